// Manufactured sources of MMS2 (test/verification/MMS2/UserSources.H):
// with x along the longest box direction and the exact profiles
//   n_e = E_eps = x^3/alpha + n0, n_i = x^3/(2 alpha) + n0,
//   E = -(5x^4 - 1)/40, Te = (2/3)(E_eps/n_e)/kB,
// each equation receives d(Gamma)/dx minus the ionization term evaluated
// on the exact solution (with the actual neutral density), and the energy
// equation the divergence of its 5/3-scaled flux minus the Joule term plus
// the inelastic (4 J per ionization) and elastic losses.
#pragma once
#include "vd_vars.H"

namespace user_sources {
AMREX_GPU_DEVICE AMREX_INLINE int mms2_bigdir(vd::GpuArray<vd::Real, 3> lo,
                                              vd::GpuArray<vd::Real, 3> hi)
{
    // the reference picks the last of the directions whose length equals
    // the maximum
    vd::Real mx = hi[0] - lo[0];
    for (int d = 1; d < 3; ++d) mx = std::max(mx, hi[d] - lo[d]);
    int big = 0;
    for (int d = 0; d < 3; ++d)
        if (hi[d] - lo[d] == mx) big = d;
    return big;
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_react_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& rxnsrc,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm,
    vd::Real Tg, vd::Real Pg)
{
    using vd::Real;
    const int b = mms2_bigdir(prob_lo, prob_hi);
    const int iv[3] = {i, j, k};
    const Real x = prob_lo[b] + (iv[b] + 0.5) * dx[b];
    const Real n0 = prob_parm.n0;
    const Real alpha = ECHARGE / EPS0;
    const Real x2 = x * x, x3 = x * x * x;
    const Real Ee = x3 / alpha + n0;
    const Real ne = x3 / alpha + n0;
    const Real dne = 3.0 * x2 / alpha;
    const Real d2ne = 6.0 * x / alpha;
    const Real ni = x3 / (2.0 * alpha) + n0;
    const Real dni = 3.0 * x2 / (2.0 * alpha);
    const Real d2ni = 6.0 * x / (2.0 * alpha);
    const Real E = (-1 / 40.0) * (5 * x * x * x * x - 1.0);
    const Real dE = -x3 / 2.0;
    const Real Te = (2.0 / 3.0) * (Ee / ne) / K_B;
    const Real Ta = 2.0 / K_B;
    const Real mue = -1.0, De = 1.0, mui = 0.5, Di = 0.5;
    const Real gam_e = mue * ne * E - De * dne;
    const Real dgam_e = mue * dne * E + mue * ne * dE - De * d2ne;
    const Real dgam_een = (5.0 / 3.0) * dgam_e;
    const Real dgam_i = mui * dni * E + mui * ni * dE - Di * d2ni;
    const Real iz = 5.0 * std::exp(-Ta / Te) * ne * phi(i, j, k, HE_ID);
    rxnsrc(i, j, k, E_ID) += (dgam_e - iz);
    rxnsrc(i, j, k, HEp_ID) += (dgam_i - iz);
    const Real joule = -ECHARGE * gam_e * E;
    const Real inel = 4.0 * iz;
    const Real nu = 10000.0;
    const Real elas = 3.0 / 2.0 * K_B * ne * (Te - Tg) * nu * (2.0 * ME / (4.0 * M_AMU));
    rxnsrc(i, j, k, EEN_ID) += (dgam_een - joule + inel + elas);
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_potential_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& source,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm)
{
}
} // namespace user_sources
