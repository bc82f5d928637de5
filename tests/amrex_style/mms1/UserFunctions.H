#ifndef MMS1_AMREX_USERFUNCTIONS_H
#define MMS1_AMREX_USERFUNCTIONS_H
#include <AMReX_Geometry.H>
#include <AMReX_FArrayBox.H>
#include <Chemistry.H>
#include <ProbParm.H>

// Dirichlet data through Robin a = 1, b = 0: the potential 0 at both ends,
// NI 0 at the low end and 1 at the high end; drift only along the axial
// direction and only for NI.  The integrated-current arguments are unused.
namespace user_transport {
using namespace amrex;

AMREX_GPU_DEVICE AMREX_INLINE void potential_bc(
    int i, int j, int k, int dir, int sgn, Array4<Real> const& phi,
    Array4<Real> const& bc_arr, Array4<Real> const& robin_a, Array4<Real> const& robin_b,
    Array4<Real> const& robin_f, GpuArray<Real, AMREX_SPACEDIM> prob_lo,
    GpuArray<Real, AMREX_SPACEDIM> prob_hi, GpuArray<Real, AMREX_SPACEDIM> dx,
    const Real time, ProbParm const& prob_parm, amrex::Real Tg, amrex::Real Pg,
    amrex::Real app_voltage, GpuArray<Real, MAX_CURRENT_LOCS> int_currents,
    GpuArray<Real, MAX_CURRENT_LOCS> int_current_areas,
    GpuArray<int, MAX_CURRENT_LOCS> int_current_surfaces)
{
    IntVect ghost_cell{AMREX_D_DECL(i, j, k)};
    if (sgn == -1) ghost_cell[dir] -= 1;
    robin_a(ghost_cell) = 1.0;
    robin_b(ghost_cell) = 0.0;
    robin_f(ghost_cell) = 0.0;
}

AMREX_GPU_DEVICE AMREX_INLINE void species_bc(
    int i, int j, int k, int dir, int sgn, int spec_id, int bcspec_id,
    Array4<Real> const& phi, Array4<Real> const& bc_arr, Array4<Real> const& robin_a,
    Array4<Real> const& robin_b, Array4<Real> const& robin_f,
    GpuArray<Real, AMREX_SPACEDIM> prob_lo, GpuArray<Real, AMREX_SPACEDIM> prob_hi,
    GpuArray<Real, AMREX_SPACEDIM> dx, const Real time, ProbParm const& prob_parm,
    amrex::Real Tg, amrex::Real Pg, GpuArray<Real, MAX_CURRENT_LOCS> int_currents,
    GpuArray<Real, MAX_CURRENT_LOCS> int_current_areas,
    GpuArray<int, MAX_CURRENT_LOCS> int_current_surfaces)
{
    IntVect ghost_cell{AMREX_D_DECL(i, j, k)};
    if (sgn == -1) ghost_cell[dir] -= 1;
    const Real v = (sgn == -1) ? 0.0 : 1.0;
    robin_a(ghost_cell, bcspec_id) = 1.0;
    robin_b(ghost_cell, bcspec_id) = 0.0;
    robin_f(ghost_cell, bcspec_id) = v;
    bc_arr(ghost_cell, bcspec_id) = v;
}

AMREX_GPU_DEVICE AMREX_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4<Real> const& phi,
    GpuArray<Real, AMREX_SPACEDIM> dx, const Real time, ProbParm const& prob_parm,
    amrex::Real Tg, amrex::Real Pg)
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
#endif
