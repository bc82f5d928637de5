// Linear advection case of the reference (test/verification/Advect): a
// neutral species AR carried at a prescribed velocity by the WENO5 drift
// flux, periodic boundaries, no diffusion; initial AR = sin(pi x - sin(pi x)/pi)
// (Ghosh & Baeder 2014), exact solution the initial profile shifted by v t
// (test/verification/Advect/get_error_1d.py).
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define AR_ID 1
#define NUM_SPECIES 2
#define NUM_IONS 0
#define FIRST_ION 0
#define NUM_NEUTRALS 1
#define FIRST_NEUTRAL 1
#define NUM_REACTIONS 1

inline void CKSYMS_STR(std::vector<std::string>& kname) { kname = {"E", "AR"}; }

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    return n == 0 ? 0.000549 : 39.948;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[0] = -1;
    kcharge[1] = 0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return -1.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specDiff(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const vd::Real T, vd::Real C[], vd::Real wdot[], const vd::Real Te, const vd::Real EN,
    vd::Real* ener_exch)
{
    for (int i = 0; i < NUM_SPECIES; ++i) wdot[i] = 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 5802.25;
}
