// Prescribed advection velocity of AR; boundaries are periodic, so the
// boundary callbacks are never reached.
#pragma once
#include "vd_vars.H"
#define VD_HAS_USER_TRANSPORT 1

namespace user_transport {
using vd::Array4;
using vd::GpuArray;
using vd::IntVect;
using vd::Real;

AMREX_GPU_DEVICE AMREX_INLINE void potential_bc(
    int i, int j, int k, int dir, int sgn, Array4 const& phi, Array4 const& bcarr,
    Array4 const& robin_a, Array4 const& robin_b, Array4 const& robin_f,
    GpuArray<Real, 3> prob_lo, GpuArray<Real, 3> prob_hi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg, Real app_voltage)
{
}

AMREX_GPU_DEVICE AMREX_INLINE void species_bc(
    int i, int j, int k, int dir, int sgn, int spec_id, int bcspec_id, Array4 const& phi,
    Array4 const& bc_arr, Array4 const& robin_a, Array4 const& robin_b,
    Array4 const& robin_f, GpuArray<Real, 3> prob_lo, GpuArray<Real, 3> prob_hi,
    GpuArray<Real, 3> dx, const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    const Real vel[3] = {prob_parm.velx, prob_parm.vely, prob_parm.velz};
    return (specid == AR_ID) ? vel[dir] : 0.0;
}
} // namespace user_transport
