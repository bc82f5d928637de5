// Initial data of MMS3 (test/verification/MMS3/Prob.H): electrons, the ion
// and the electron energy n0 (1 + sin(pi x / L)) along the axial direction,
// the background neutral 1 m^-3, Te 0.666, everything else 0.
#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.query("axial_dir", h_prob_parm.axdir);
}

AMREX_GPU_HOST_DEVICE AMREX_INLINE void initdomaindata(
    vd::Box const& bx, vd::Array4 const& phi, vd::GeometryData const& geomdata,
    ProbParm const* prob_parm)
{
    const vd::Real* plo = geomdata.ProbLo();
    const vd::Real* phi_ = geomdata.ProbHi();
    const vd::Real* dx = geomdata.CellSize();
    const int a = prob_parm->axdir;
    const vd::Real len = phi_[a] - plo[a];
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
            {
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 0.0;
                phi(i, j, k, CMASK_ID) = 1.0;
                const int iv[3] = {i, j, k};
                const vd::Real x = plo[a] + (0.5 + iv[a]) * dx[a];
                const vd::Real prof = prob_parm->n0 * (1 + std::sin(PI * x / len));
                phi(i, j, k, E_ID) = prof;
                phi(i, j, k, HE_ID) = 1.0;
                phi(i, j, k, HEp_ID) = prof;
                phi(i, j, k, EEN_ID) = prof;
                phi(i, j, k, ETEMP_ID) = 0.666;
            }
}
