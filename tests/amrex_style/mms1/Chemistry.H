// MMS1 written the way a reference case directory is: AMReX headers and
// types, species names in Chemistry.cpp.  One drifting, diffusing negative
// species NI (mu = -1, D = 1) coupled to the Poisson equation; electrons
// inert.  A test fixture for the compatibility headers (vidyut_b200/compat):
// built unchanged, it must give the bits of vidyut_b200/cases/mms1.
#ifndef MMS1_AMREX_CHEMISTRY_H
#define MMS1_AMREX_CHEMISTRY_H
#include <AMReX_Gpu.H>
#include <AMReX_REAL.H>
#include <VarDefines.H>
#include <UnivConstants.H>
#include <string>

#define E_ID 0
#define NI_ID 1
#define NUM_SPECIES 2
#define FIRST_ION 1
#define NUM_IONS 1
#define FIRST_NEUTRAL 0
#define NUM_NEUTRALS 0
#define NUM_REACTIONS 1

void CKSYMS_STR(amrex::Vector<std::string>& kname);

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real mw(const int n)
{
    const amrex::Real w[NUM_SPECIES] = {0.000549, 39.948};
    return w[n];
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[E_ID] = -1;
    kcharge[NI_ID] = -1;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real specMob(
    const int specid, const amrex::Real Te, const amrex::Real ndens, const amrex::Real emag,
    const amrex::Real T)
{
    return -1.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real specDiff(
    const int specid, const amrex::Real Te, const amrex::Real ndens, const amrex::Real emag,
    const amrex::Real T)
{
    amrex::Real d = 0.0;
    if (specid == NI_ID) d = 1.0;
    return d;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const amrex::Real T, amrex::Real C[], amrex::Real wdot[], const amrex::Real Te,
    const amrex::Real EN, amrex::Real* ener_exch)
{
    for (int sp = 0; sp < NUM_SPECIES; ++sp) wdot[sp] = 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real
etempLFA(const amrex::Real Tg, amrex::Real C[], const amrex::Real EN)
{
    return 5802.25;
}
#endif
