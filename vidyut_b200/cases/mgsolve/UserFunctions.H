// Boundary callbacks of the solver workload.  With user_defined_potential
// off (the default) the workload uses the default callbacks: Dirichlet 0 V
// on the z faces, Neumann on x and y.  With it on and Robin (4) potential
// sides on z, the potential sees an electrode layout of a sputter reactor
// (the geometry of the reference's test/models/Ar_RF_Sputter3d potential
// callback, here on the unit cube): in the low-z wall two disc electrodes
// of radius prob.trode_rad centred at (1/2, 1/2 -+ prob.trode_sep) held at
// +-prob.trode_volt through Robin (a, b, f) = (1, 0, V); in the high-z wall
// a grounded disc substrate of radius prob.subs_rad at the centre; every
// other boundary face (a, b, f) = (0, 1, 0), insulating.  A wall of
// Dirichlet patches in a Neumann face is the case the multigrid hierarchy's
// Robin coarsening has to keep: its coarse faces must not turn Neumann.
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
    bcarr(ghost) = 0.0;
    Real a = 0.0, b = 1.0, f = 0.0;
    if (dir == 2)
    {
        // face centre in the (x, y) plane of the wall
        const Real x = prob_lo[0] + (i + 0.5) * dx[0] - 0.5 * (prob_lo[0] + prob_hi[0]);
        const Real y = prob_lo[1] + (j + 0.5) * dx[1] - 0.5 * (prob_lo[1] + prob_hi[1]);
        const Real r1 = prob_parm.trode_rad, rs = prob_parm.subs_rad;
        const Real s = prob_parm.trode_sep;
        if (sgn == -1)
        {
            if (x * x + (y + s) * (y + s) < r1 * r1)
            {
                a = 1.0; b = 0.0; f = prob_parm.trode_volt;
            }
            else if (x * x + (y - s) * (y - s) < r1 * r1)
            {
                a = 1.0; b = 0.0; f = -prob_parm.trode_volt;
            }
        }
        else if (x * x + y * y < rs * rs)
        {
            a = 1.0; b = 0.0; f = 0.0;
        }
    }
    robin_a(ghost) = a;
    robin_b(ghost) = b;
    robin_f(ghost) = f;
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
    bc_arr(ghost, bcspec_id) = 0.0;
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi, GpuArray<Real, 3> dx,
    const Real time, ProbParm const& prob_parm, Real Tg, Real Pg)
{
    return 0.0;
}
} // namespace user_transport
