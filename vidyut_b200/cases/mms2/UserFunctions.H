// Boundary and velocity callbacks of MMS2 (test/verification/MMS2/
// UserFunctions.H): the potential is Dirichlet 0 through Robin a=1, b=0,
// f=0 on every non-periodic face; electrons, the ion and the electron
// energy carry the exact solution's Dirichlet values in the boundary array
// (n0 on the low faces; 1/alpha + n0 for electrons and energy and
// 1/(2 alpha) + n0 for the ion on the high faces); drift only along the
// axial direction, with the mobility at a dummy total density of 1.
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
    const Real n0 = prob_parm.n0;
    const Real alpha = ECHARGE / EPS0;
    const bool carried = spec_id == E_ID || spec_id == HEp_ID || spec_id == EEN_ID;
    if (!carried) return;
    if (sgn == -1)
        bc_arr(ghost, bcspec_id) = 0.0 + n0;
    else if (spec_id == HEp_ID)
        bc_arr(ghost, bcspec_id) = 1.0 / (2.0 * alpha) + n0;
    else
        bc_arr(ghost, bcspec_id) = 1.0 / alpha + n0;
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    if (dir != prob_parm.axdir) return 0.0;
    const Real ex = phi(cellid, EFX_ID), ey = phi(cellid, EFY_ID), ez = phi(cellid, EFZ_ID);
    const Real emag = std::sqrt(ex * ex + ey * ey + ez * ez);
    const Real mu = specMob(specid, phi(cellid, ETEMP_ID), 1.0, emag, Tg);
    return mu * phi(cellid, EFX_ID + dir);
}
} // namespace user_transport
