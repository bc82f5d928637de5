// Initial data of MMS2 (test/verification/MMS2/Prob.H): every component
// 1e-12, then a fraction `solnfrac` of the exact profiles along the axial
// direction (electrons with a 1e-5 n0 twiddle so that they are not zero),
// neutral density 1, electron temperature 1, cell mask 0 outside [0, 1].
#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.query("axial_dir", h_prob_parm.axdir);
    pp.query("solnfrac", h_prob_parm.solnfrac);
}

AMREX_GPU_HOST_DEVICE AMREX_INLINE void initdomaindata(
    vd::Box const& bx, vd::Array4 const& phi, vd::GeometryData const& geomdata,
    ProbParm const* prob_parm)
{
    const vd::Real* plo = geomdata.ProbLo();
    const vd::Real* dx = geomdata.CellSize();
    const int a = prob_parm->axdir;
    const vd::Real alpha = ECHARGE / EPS0;
    const vd::Real f = prob_parm->solnfrac;
    const vd::Real n0 = prob_parm->n0;
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
            {
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 1e-12;
                const int iv[3] = {i, j, k};
                const vd::Real x = plo[a] + (0.5 + iv[a]) * dx[a];
                phi(i, j, k, CMASK_ID) = (x * (x - 1.0) > 0.0) ? 0.0 : 1.0;
                phi(i, j, k, E_ID) = f * (x * x * x / alpha + n0) + 1e-5 * n0;
                phi(i, j, k, HE_ID) = 1.0;
                phi(i, j, k, HEp_ID) = f * (x * x * x / (2.0 * alpha) + n0);
                phi(i, j, k, POT_ID) = f * (1.0 / 24.0) * (x * x * x * x * x - x);
                phi(i, j, k, EFX_ID) = 0.0;
                phi(i, j, k, EFY_ID) = 0.0;
                phi(i, j, k, EFZ_ID) = 0.0;
                phi(i, j, k, EEN_ID) = f * (x * x * x / alpha + n0);
                phi(i, j, k, ETEMP_ID) = 1.0;
            }
}
