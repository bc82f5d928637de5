// No user sources in the solver workload.
#pragma once
#include "vd_vars.H"

namespace user_sources {
AMREX_GPU_DEVICE AMREX_INLINE void add_user_react_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& rxnsrc,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm,
    vd::Real Tg, vd::Real Pg)
{
}

AMREX_GPU_DEVICE AMREX_INLINE void add_user_potential_sources(
    int i, int j, int k, vd::Array4 const& phi, vd::Array4 const& source,
    vd::GpuArray<vd::Real, 3> prob_lo, vd::GpuArray<vd::Real, 3> prob_hi,
    vd::GpuArray<vd::Real, 3> dx, const vd::Real time, ProbParm const& prob_parm)
{
}
} // namespace user_sources
#define VD_NO_USER_REACT_SOURCES 1
#define VD_NO_USER_POTENTIAL_SOURCES 1
