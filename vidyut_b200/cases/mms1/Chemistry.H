// Method-of-manufactured-solutions case 1 of the reference
// (test/verification/MMS1): one drifting, diffusing negative species NI
// coupled to the Poisson equation,
//   dn/dt + d(mu n E)/dx = d/dx(D dn/dx) + (5x^4/3 - x/6 - 2),  n(0)=0, n(1)=1
//   d2phi/dx2 = n,  phi(0) = phi(1) = 0,  mu = -1, D = 1,
// with exact steady solution n = x^2, phi = (x^4 - x)/12
// (test/verification/MMS1/README.md).  Electrons are present but inert.
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define NI_ID 1
#define NUM_SPECIES 2
#define FIRST_ION 1
#define NUM_IONS 1
#define FIRST_NEUTRAL 0
#define NUM_NEUTRALS 0
#define NUM_REACTIONS 1

inline void CKSYMS_STR(std::vector<std::string>& kname) { kname = {"E", "NI"}; }

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    return n == 0 ? 0.000549 : 39.948;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[0] = -1;
    kcharge[1] = -1;
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
    return (specid == NI_ID) ? 1.0 : 0.0;
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
