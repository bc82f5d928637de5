// Boundary and velocity callbacks of MMS3 (test/verification/MMS3/
// UserFunctions.H): Dirichlet 0 for the potential through Robin a=1, b=0;
// species walls in homogeneous-Robin form (a=0, b=1) with n0 in the boundary
// array on the low faces; drift only along the axial direction (the
// mobilities are zero, so none takes place).
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
    if (sgn == -1) ghost[dir] -= 1;
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
    if (sgn == -1) ghost[dir] -= 1;
    robin_a(ghost, bcspec_id) = 0.0;
    robin_b(ghost, bcspec_id) = 1.0;
    robin_f(ghost, bcspec_id) = 0.0;
    if (sgn == -1 && (spec_id == E_ID || spec_id == HEp_ID || spec_id == EEN_ID))
        bc_arr(ghost, bcspec_id) = 0.0 + prob_parm.n0;
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    if (dir != prob_parm.axdir) return 0.0;
    const Real ex = phi(cellid, EFX_ID), ey = phi(cellid, EFY_ID), ez = phi(cellid, EFZ_ID);
    const Real emag = std::sqrt(ex * ex + ey * ey + ez * ez);
    return specMob(specid, phi(cellid, ETEMP_ID), 1.0, emag, Tg) * phi(cellid, EFX_ID + dir);
}
} // namespace user_transport
