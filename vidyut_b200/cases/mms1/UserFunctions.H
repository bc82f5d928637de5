// Boundary and velocity callbacks of the MMS1 case: Dirichlet data through
// Robin a=1, b=0 on the potential (0 at both ends) and on NI (0 low, 1 high);
// drift only along the axial direction and only for NI.
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
    IntVect ghost{i, j, k};
    ghost[dir] += (sgn == -1) ? -1 : 0;
    robin_a(ghost) = 1.0;
    robin_b(ghost) = 0.0;
    robin_f(ghost) = 0.0;
}

AMREX_GPU_DEVICE AMREX_INLINE void species_bc(
    int i, int j, int k, int dir, int sgn, int spec_id, int bcspec_id, Array4 const& phi,
    Array4 const& bc_arr, Array4 const& robin_a, Array4 const& robin_b,
    Array4 const& robin_f, GpuArray<Real, 3> prob_lo, GpuArray<Real, 3> prob_hi,
    GpuArray<Real, 3> dx, const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    IntVect ghost{i, j, k};
    ghost[dir] += (sgn == -1) ? -1 : 0;
    const Real v = (sgn == -1) ? 0.0 : 1.0;
    robin_a(ghost, bcspec_id) = 1.0;
    robin_b(ghost, bcspec_id) = 0.0;
    robin_f(ghost, bcspec_id) = v;
    bc_arr(ghost, bcspec_id) = v;
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    Real vel = 0.0;
    if (dir == prob_parm.axdir && specid == NI_ID)
    {
        const Real ex = phi(cellid, EFX_ID), ey = phi(cellid, EFY_ID), ez = phi(cellid, EFZ_ID);
        const Real emag = std::sqrt(ex * ex + ey * ey + ez * ez);
        const Real mu = specMob(specid, phi(cellid, ETEMP_ID), 1.0, emag, Tg);
        vel = mu * phi(cellid, EFX_ID + dir);
    }
    return vel;
}
} // namespace user_transport
