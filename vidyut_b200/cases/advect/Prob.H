#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.query("one_dim", h_prob_parm.one_dim);
    pp.query("blobrad", h_prob_parm.blobrad);
    pp.query("velx", h_prob_parm.velx);
    pp.query("vely", h_prob_parm.vely);
    pp.query("velz", h_prob_parm.velz);
}

AMREX_GPU_HOST_DEVICE AMREX_INLINE void initdomaindata(
    vd::Box const& bx, vd::Array4 const& phi, vd::GeometryData const& geomdata,
    ProbParm const* prob_parm)
{
    const vd::Real* lo = geomdata.ProbLo();
    const vd::Real* hi = geomdata.ProbHi();
    const vd::Real* dx = geomdata.CellSize();
    const vd::Real midx = 0.5 * (lo[0] + hi[0]), midy = 0.5 * (lo[1] + hi[1]);
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
            {
                const vd::Real x = lo[0] + (0.5 + i) * dx[0];
                const vd::Real y = lo[1] + (0.5 + j) * dx[1];
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 0.0;
                phi(i, j, k, CMASK_ID) = 1.0;
                if (prob_parm->one_dim)
                    phi(i, j, k, AR_ID) = std::sin(PI * x - std::sin(PI * x) / PI);
                else
                    phi(i, j, k, AR_ID) =
                        std::exp(-0.25 * ((x - midx) * (x - midx) + (y - midy) * (y - midy)) /
                                 prob_parm->blobrad / prob_parm->blobrad);
                phi(i, j, k, ETEMP_ID) = 0.5 * eV;
            }
}
