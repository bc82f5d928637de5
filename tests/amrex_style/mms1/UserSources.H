#ifndef MMS1_AMREX_USERSOURCES_H
#define MMS1_AMREX_USERSOURCES_H
#include <AMReX_Geometry.H>
#include <AMReX_FArrayBox.H>
#include <Chemistry.H>
#include <ProbParm.H>

// Manufactured sources: 5x^4/3 - x/6 - 2 for NI and +n_NI on the Poisson
// right-hand side, x along the longest box direction.
namespace user_sources {
using namespace amrex;

AMREX_GPU_DEVICE AMREX_INLINE int longest_dir(GpuArray<Real, AMREX_SPACEDIM> lo,
                                              GpuArray<Real, AMREX_SPACEDIM> hi)
{
    int big = 0;
    Real len = hi[0] - lo[0];
    for (int d = 1; d < AMREX_SPACEDIM; ++d)
        if (hi[d] - lo[d] > len)
        {
            len = hi[d] - lo[d];
            big = d;
        }
    return big;
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_react_sources(
    int i, int j, int k, Array4<Real> const& phi, Array4<Real> const& rxnsrc,
    GpuArray<Real, AMREX_SPACEDIM> prob_lo, GpuArray<Real, AMREX_SPACEDIM> prob_hi,
    GpuArray<Real, AMREX_SPACEDIM> dx, const Real time, ProbParm const& prob_parm,
    amrex::Real Tg, amrex::Real Pg)
{
    const int b = longest_dir(prob_lo, prob_hi);
    const int iv[3] = {i, j, k};
    const Real x = prob_lo[b] + (iv[b] + 0.5) * dx[b];
    rxnsrc(i, j, k, NI_ID) += 5.0 * x * x * x * x / 3.0 - x / 6.0 - 2.0;
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_potential_sources(
    int i, int j, int k, Array4<Real> const& phi, Array4<Real> const& source,
    GpuArray<Real, AMREX_SPACEDIM> prob_lo, GpuArray<Real, AMREX_SPACEDIM> prob_hi,
    GpuArray<Real, AMREX_SPACEDIM> dx, const Real time, ProbParm const& prob_parm)
{
    source(i, j, k) += phi(i, j, k, NI_ID);
}
} // namespace user_sources
#endif
