// CPU ORACLE -- test infrastructure only.
//
// The oracle's own restatement of the reference's default transport and
// boundary callbacks (Source/PlasmaChem.H:16-280, namespace
// plasmachem_transport) and of plasmachem::get_charge
// (Source/PlasmaChem.cpp:33).  It is written separately from the library's
// copy (vidyut_b200/csrc/PlasmaChem.H) so that a misreading of the
// reference on either side shows up as a parity failure instead of being
// compared with itself.  Case hook headers (Chemistry.H, UserFunctions.H,
// ...) are plugin inputs and are shared with the library.
//
// Conventions of the reference's callbacks: (i,j,k) is a boundary face
// index along `dir`; sgn = -1 on the low side, +1 on the high side; the
// ghost cell is the face index minus one on the low side and the face index
// itself on the high side; the interior cell is the other neighbour.
#pragma once

#include "vd_vars.H"

namespace plasmachem {
inline int get_charge(int specid)
{
    int z[NUM_SPECIES];
    CKCHRG(z);
    return z[specid];
}
} // namespace plasmachem

namespace plasmachem_transport {

namespace detail {
struct Sides
{
    vd::IntVect ghost, inner;
};
inline Sides sides_of(int i, int j, int k, int dir, int sgn)
{
    Sides s{{i, j, k}, {i, j, k}};
    if (sgn < 0)
        s.ghost[dir] -= 1; // low side: ghost below the face
    else
        s.inner[dir] -= 1; // high side: interior cell below the face
    return s;
}
inline vd::Real field_magnitude(vd::Array4 const& a, vd::IntVect c)
{
    vd::Real m2 = 0.0;
    for (int d = 0; d < 3; ++d) m2 += a(c, EFX_ID + d) * a(c, EFX_ID + d);
    return std::sqrt(m2);
}
inline vd::Real total_density(vd::Array4 const& a, vd::IntVect c)
{
    vd::Real t = 0.0;
    for (int s = 0; s < NUM_SPECIES; ++s) t += a(c, s);
    return t;
}
// one-sided thermal flux n cbar / 4 with cbar = sqrt(8 kB T / pi / m),
// evaluated in the reference's operation order
inline vd::Real thermal_flux(vd::Real n, vd::Real T, vd::Real m)
{
    const vd::Real cbar = std::sqrt(8.0 * K_B * T / PI / m);
    return n * cbar / 4.0;
}
} // namespace detail

// Source/PlasmaChem.H:16-73: Dirichlet app_voltage on every non-periodic
// face (the reference's lo and hi branches set the same values).
inline void potential_bc(int i, int j, int k, int dir, int sgn, vd::Array4 const& phi,
                         vd::Array4 const& bc_arr, vd::Array4 const& robin_a,
                         vd::Array4 const& robin_b, vd::Array4 const& robin_f,
                         vd::GpuArray<vd::Real, 3>, vd::GpuArray<vd::Real, 3>,
                         vd::GpuArray<vd::Real, 3>, const vd::Real, ProbParm const&, vd::Real,
                         vd::Real, vd::Real app_voltage)
{
    const vd::IntVect g = detail::sides_of(i, j, k, dir, sgn).ghost;
    robin_a(g) = 1.0;
    robin_b(g) = 0.0;
    robin_f(g) = app_voltage;
    bc_arr(g) = app_voltage;
}

// Source/PlasmaChem.H:75-200: homogeneous-Robin form (a=0, b=1, f=0) with
// the inhomogeneous Neumann value -flux/D in bc_arr, the flux being
//   electrons:        thermal flux of n_e at Te, times sgn;
//   electron energy:  2 kB Te times the electron thermal flux, times sgn;
//   charged heavies:  the drift flux mu n E_dir where it points out of the
//                     domain (mu n E_dir sgn >= 0), else zero;
//   neutrals:         thermal flux at Tg with the species mass mw*M_AMU of
//                     the density at the face index itself (the reference
//                     reads phi(i,j,k), the ghost cell on the high side).
inline void species_bc(int i, int j, int k, int dir, int sgn, int spec_id, int bcspec_id,
                       vd::Array4 const& phi, vd::Array4 const& bc_arr,
                       vd::Array4 const& robin_a, vd::Array4 const& robin_b,
                       vd::Array4 const& robin_f, vd::GpuArray<vd::Real, 3>,
                       vd::GpuArray<vd::Real, 3>, vd::GpuArray<vd::Real, 3>, const vd::Real,
                       ProbParm const&, vd::Real Tg, vd::Real)
{
    const detail::Sides s = detail::sides_of(i, j, k, dir, sgn);
    robin_a(s.ghost, bcspec_id) = 0.0;
    robin_b(s.ghost, bcspec_id) = 1.0;
    robin_f(s.ghost, bcspec_id) = 0.0;
    const vd::Real te = phi(s.inner, ETEMP_ID);
    const vd::Real nt = detail::total_density(phi, s.inner);
    const vd::Real em = detail::field_magnitude(phi, s.inner);
    const vd::Real D = specDiff(spec_id, te, nt, em, Tg);
    vd::Real flux = 0.0;
    if (spec_id == E_ID)
        flux = detail::thermal_flux(phi(s.inner, E_ID), te, ME) * sgn;
    else if (spec_id == EEN_ID)
        flux = (2.0 * K_B * te) * detail::thermal_flux(phi(s.inner, E_ID), te, ME) * sgn;
    else if (plasmachem::get_charge(spec_id) != 0)
    {
        const vd::Real drift =
            specMob(spec_id, te, nt, em, Tg) * phi(s.inner, spec_id) * phi(s.inner, EFX_ID + dir);
        bc_arr(s.ghost, bcspec_id) = (drift * sgn >= 0.0) ? -drift / D : 0.0;
        return;
    } else
        flux = detail::thermal_flux(phi(i, j, k, spec_id), Tg, mw(spec_id) * M_AMU) * sgn;
    bc_arr(s.ghost, bcspec_id) = -flux / D;
}

// Source/PlasmaChem.H:257-280: v = mu(Te, n_total, |E|) E_dir.
inline vd::Real compute_vel(vd::IntVect cellid, int dir, int specid, vd::Array4 const& phi,
                            vd::GpuArray<vd::Real, 3>, const vd::Real, ProbParm const&,
                            vd::Real Tg, vd::Real)
{
    const vd::Real mu = specMob(specid, phi(cellid, ETEMP_ID), detail::total_density(phi, cellid),
                                detail::field_magnitude(phi, cellid), Tg);
    return mu * phi(cellid, EFX_ID + dir);
}

} // namespace plasmachem_transport
