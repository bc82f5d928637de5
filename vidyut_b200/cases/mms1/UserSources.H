// Manufactured sources of MMS1: the NI source and +n_NI on the Poisson
// right-hand side, with x measured along the longest box direction.
#pragma once
#include "vd_vars.H"

namespace user_sources {
AMREX_GPU_DEVICE AMREX_INLINE int mms_bigdir(vd::GpuArray<vd::Real, 3> lo,
                                             vd::GpuArray<vd::Real, 3> hi)
{
    int big = 0;
    vd::Real len = hi[0] - lo[0];
    for (int d = 1; d < 3; ++d)
        if (hi[d] - lo[d] > len)
        {
            len = hi[d] - lo[d];
            big = d;
        }
    return big;
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_react_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& rxnsrc,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm,
    vd::Real Tg, vd::Real Pg)
{
    const int b = mms_bigdir(prob_lo, prob_hi);
    const int iv[3] = {i, j, k};
    const vd::Real x = prob_lo[b] + (iv[b] + 0.5) * dx[b];
    rxnsrc(i, j, k, NI_ID) += 5.0 * x * x * x * x / 3.0 - x / 6.0 - 2.0;
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_potential_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& source,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm)
{
    source(i, j, k) += phi(i, j, k, NI_ID);
}
} // namespace user_sources
