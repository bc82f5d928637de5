#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.queryarr("n0", h_prob_parm.n0, 8);
    pp.query("te", h_prob_parm.te);
}

AMREX_GPU_HOST_DEVICE AMREX_INLINE void initdomaindata(
    vd::Box const& bx, vd::Array4 const& phi, vd::GeometryData const& geomdata,
    ProbParm const* prob_parm)
{
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
            {
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 0.0;
                phi(i, j, k, CMASK_ID) = 1.0;
                for (int s = 0; s < NUM_SPECIES; ++s) phi(i, j, k, s) = prob_parm->n0[s];
                phi(i, j, k, ETEMP_ID) = prob_parm->te;
                phi(i, j, k, EEN_ID) = 1.5 * prob_parm->n0[E_ID] * K_B * prob_parm->te;
            }
}
