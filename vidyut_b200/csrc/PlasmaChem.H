// Default transport and boundary callbacks, used when a case leaves
// vidyut.user_defined_{potential,species,vel} at 0.  Behaviour follows the
// reference's plasmachem_transport namespace (Source/PlasmaChem.H:16-280) and
// plasmachem::get_charge (Source/PlasmaChem.cpp:33).
//
// Boundary callbacks receive the index of a boundary FACE (i,j,k) in the
// normal direction `dir` and the outward sign `sgn` (-1 low side, +1 high
// side).  The ghost cell is (face-1) on the low side and (face) on the high
// side; the adjacent interior cell is (face) on the low side and (face-1) on
// the high side.  `bc_arr`, `robin_a/b/f` are views whose only valid
// entries are those ghost cells.
#pragma once

#include "vd_vars.H"

namespace plasmachem {
VD_HD VD_INLINE int get_charge(int specid)
{
    int q[NUM_SPECIES];
    CKCHRG(q);
    return q[specid];
}
} // namespace plasmachem

namespace plasmachem_transport {

using vd::Array4;
using vd::GpuArray;
using vd::IntVect;
using vd::Real;

// Dirichlet value app_voltage on every non-periodic potential face
// (Source/PlasmaChem.H:16-73).
VD_HD VD_INLINE void potential_bc(
    int i, int j, int k, int dir, int sgn, Array4 const& phi,
    Array4 const& bc_arr, Array4 const& robin_a, Array4 const& robin_b,
    Array4 const& robin_f, GpuArray<Real, 3> prob_lo,
    GpuArray<Real, 3> prob_hi, GpuArray<Real, 3> dx, const Real time,
    ProbParm const& prob_parm, Real Tg, Real Pg, Real app_voltage)
{
    IntVect ghost{i, j, k};
    ghost[dir] += (sgn == -1) ? -1 : 0;
    robin_a(ghost) = 1.0;
    robin_b(ghost) = 0.0;
    robin_f(ghost) = app_voltage;
    bc_arr(ghost) = app_voltage;
}

// Wall fluxes (Source/PlasmaChem.H:75-200): electrons and electron energy
// leave at the thermal speed, charged heavies at their drift speed when the
// drift points into the wall, neutrals at their thermal speed.  The value
// stored is the normal gradient -flux/D that an inhomogeneous-Neumann
// condition imposes.
VD_HD VD_INLINE void species_bc(
    int i, int j, int k, int dir, int sgn, int spec_id, int bcspec_id,
    Array4 const& phi, Array4 const& bc_arr, Array4 const& robin_a,
    Array4 const& robin_b, Array4 const& robin_f, GpuArray<Real, 3> prob_lo,
    GpuArray<Real, 3> prob_hi, GpuArray<Real, 3> dx, const Real time,
    ProbParm const& prob_parm, Real Tg, Real Pg)
{
    IntVect cell{i, j, k};
    IntVect ghost{i, j, k};
    ghost[dir] += (sgn == -1) ? -1 : 0;
    cell[dir] += (sgn == 1) ? -1 : 0;
    const Real nrm = Real(sgn);

    robin_a(ghost, bcspec_id) = 0.0;
    robin_b(ghost, bcspec_id) = 1.0;
    robin_f(ghost, bcspec_id) = 0.0;

    Real ndens = 0.0;
    for (int sp = 0; sp < NUM_SPECIES; sp++) ndens += phi(cell, sp);
    const Real ex = phi(cell, EFX_ID), ey = phi(cell, EFY_ID),
               ez = phi(cell, EFZ_ID);
    const Real emag = std::sqrt(ex * ex + ey * ey + ez * ez);
    const Real Te = phi(cell, ETEMP_ID);

    if (spec_id == E_ID)
    {
        const Real D = specDiff(spec_id, Te, ndens, emag, Tg);
        const Real cbar = std::sqrt(8.0 * K_B * Te / PI / ME);
        const Real flx = phi(cell, E_ID) * cbar / 4.0 * nrm;
        bc_arr(ghost, bcspec_id) = -flx / D;
    } else if (spec_id == EEN_ID)
    {
        const Real D = specDiff(spec_id, Te, ndens, emag, Tg);
        const Real cbar = std::sqrt(8.0 * K_B * Te / PI / ME);
        const Real flx = (2.0 * K_B * Te) * phi(cell, E_ID) * cbar / 4.0 * nrm;
        bc_arr(ghost, bcspec_id) = -flx / D;
    } else if (plasmachem::get_charge(spec_id) != 0)
    {
        const Real mu = specMob(spec_id, Te, ndens, emag, Tg);
        const Real D = specDiff(spec_id, Te, ndens, emag, Tg);
        const Real drift = mu * phi(cell, spec_id) * phi(cell, EFX_ID + dir);
        bc_arr(ghost, bcspec_id) = (drift * nrm >= 0.0) ? (-drift / D) : 0.0;
    } else
    {
        const Real D = specDiff(spec_id, Te, ndens, emag, Tg);
        const Real cbar = std::sqrt(8.0 * K_B * Tg / PI / (mw(spec_id) * M_AMU));
        // The reference reads the density at the face index itself here
        // (Source/PlasmaChem.H:197), i.e. the ghost cell on the high side.
        const Real flx = phi(i, j, k, spec_id) * cbar / 4.0 * nrm;
        bc_arr(ghost, bcspec_id) = -flx / D;
    }
}

// Drift velocity mu(specid) * E_dir at one cell (Source/PlasmaChem.H:257-280).
VD_HD VD_INLINE Real compute_vel(
    IntVect cellid, int dir, int specid, Array4 const& phi,
    GpuArray<Real, 3> dx, const Real time, ProbParm const& prob_parm, Real Tg,
    Real Pg)
{
    const Real ex = phi(cellid, EFX_ID), ey = phi(cellid, EFY_ID),
               ez = phi(cellid, EFZ_ID);
    const Real emag = std::sqrt(ex * ex + ey * ey + ez * ez);
    Real ndens = 0.0;
    for (int sp = 0; sp < NUM_SPECIES; sp++) ndens += phi(cellid, sp);
    const Real mu = specMob(specid, phi(cellid, ETEMP_ID), ndens, emag, Tg);
    return mu * phi(cellid, EFX_ID + dir);
}

} // namespace plasmachem_transport
