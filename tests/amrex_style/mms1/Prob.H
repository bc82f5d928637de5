#ifndef MMS1_AMREX_PROB_H
#define MMS1_AMREX_PROB_H
#include <AMReX_Geometry.H>
#include <AMReX_FArrayBox.H>
#include <AMReX_ParmParse.H>
#include <AMReX_GpuMemory.H>
#include <Chemistry.H>
#include <ProbParm.H>

AMREX_INLINE void amrex_probinit(ProbParm& h_prob_parm, ProbParm& d_prob_parm)
{
    amrex::ParmParse pp("prob");
    pp.query("axial_dir", h_prob_parm.axdir);
    amrex::Gpu::htod_memcpy(&d_prob_parm, &h_prob_parm, sizeof(ProbParm));
}

// every component 1e-12, electron temperature 0.5 eV
AMREX_GPU_DEVICE AMREX_INLINE void initdomaindata(
    amrex::Box const& bx, amrex::Array4<amrex::Real> const& phi,
    amrex::GeometryData const& geomdata, ProbParm* prob_parm)
{
    const auto lo = amrex::lbound(bx);
    const auto hi = amrex::ubound(bx);
    for (int k = lo.z; k <= hi.z; ++k)
        for (int j = lo.y; j <= hi.y; ++j)
            for (int i = lo.x; i <= hi.x; ++i)
            {
                for (int c = 0; c < NVAR; c++) phi(i, j, k, c) = 1e-12;
                phi(i, j, k, CMASK_ID) = 1.0;
                phi(i, j, k, ETEMP_ID) = 0.5 * eV;
            }
}
#endif
