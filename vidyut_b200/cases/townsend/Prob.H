// Problem set-up of the Townsend discharge case, in the shape of a
// reference Prob.H (amrex_probinit + initdomaindata).
#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.query("bg", h_prob_parm.bg);
    pp.query("ngas", h_prob_parm.ngas);
    pp.query("te", h_prob_parm.te);
    pp.query("twod", h_prob_parm.twod);
    pp.query("nblobs", h_prob_parm.nblobs);
    if (h_prob_parm.nblobs > VD_MAX_BLOBS) h_prob_parm.nblobs = VD_MAX_BLOBS;
    pp.queryarr("cx", h_prob_parm.cx, h_prob_parm.nblobs);
    pp.queryarr("cy", h_prob_parm.cy, h_prob_parm.nblobs);
    pp.queryarr("cz", h_prob_parm.cz, h_prob_parm.nblobs);
    pp.queryarr("ampl", h_prob_parm.ampl, h_prob_parm.nblobs);
    pp.queryarr("sigma", h_prob_parm.sigma, h_prob_parm.nblobs);
}

AMREX_GPU_HOST_DEVICE AMREX_INLINE void initdomaindata(
    vd::Box const& bx, vd::Array4 const& phi, vd::GeometryData const& geomdata,
    ProbParm const* prob_parm)
{
    const vd::Real* prob_lo = geomdata.ProbLo();
    const vd::Real* dx = geomdata.CellSize();
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
            {
                const vd::Real x = prob_lo[0] + (0.5 + i) * dx[0];
                const vd::Real y = prob_lo[1] + (0.5 + j) * dx[1];
                const vd::Real z = prob_lo[2] + (0.5 + k) * dx[2];
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 0.0;
                phi(i, j, k, CMASK_ID) = 1.0;
                vd::Real n = prob_parm->bg;
                for (int b = 0; b < prob_parm->nblobs; ++b)
                {
                    vd::Real d2 = (x - prob_parm->cx[b]) * (x - prob_parm->cx[b]) +
                                  (y - prob_parm->cy[b]) * (y - prob_parm->cy[b]);
                    if (!prob_parm->twod)
                        d2 += (z - prob_parm->cz[b]) * (z - prob_parm->cz[b]);
                    const vd::Real s = prob_parm->sigma[b];
                    n += prob_parm->ampl[b] * std::exp(-d2 / (2.0 * s * s));
                }
                phi(i, j, k, E_ID) = n;
                phi(i, j, k, ION_ID) = n;
                phi(i, j, k, N_ID) = prob_parm->ngas;
                phi(i, j, k, ETEMP_ID) = prob_parm->te;
                phi(i, j, k, EEN_ID) = 1.5 * n * K_B * prob_parm->te;
            }
}
