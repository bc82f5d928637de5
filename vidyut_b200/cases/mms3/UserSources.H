// Source of MMS3's energy equation (test/verification/MMS3/UserSources.H):
// -10 E_eps; the species sources come from the mechanism.
#pragma once
#include "vd_vars.H"

namespace user_sources {
AMREX_GPU_DEVICE AMREX_INLINE void add_user_react_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& rxnsrc,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm,
    vd::Real Tg, vd::Real Pg)
{
    rxnsrc(i, j, k, EEN_ID) += (-10.0 * phi(i, j, k, EEN_ID));
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_potential_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& source,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm)
{
}
} // namespace user_sources
