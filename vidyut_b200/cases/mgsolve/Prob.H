// The solver workload's state is generated on the host and copied in
// (vidyut_b200/workloads.py, mgsolve_state); initdomaindata only clears it.
// prob.* sets the electrode layout of the user potential callback.
#pragma once
#include "vd_vars.H"
#include "vd_parmparse.H"

inline void amrex_probinit(ProbParm& h_prob_parm, vd::ParmParse& pp)
{
    pp.query("trode_rad", h_prob_parm.trode_rad);
    pp.query("trode_sep", h_prob_parm.trode_sep);
    pp.query("trode_volt", h_prob_parm.trode_volt);
    pp.query("subs_rad", h_prob_parm.subs_rad);
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
            }
}
