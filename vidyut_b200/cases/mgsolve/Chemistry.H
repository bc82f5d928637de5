// Linear-solver workload (mixed-precision Poisson and implicit diffusion on
// a unit cube): electrons and one positive ion carry a net charge density
// n_ion - n_e, and the ion diffuses with a per-cell diffusivity.  No
// reactions and no drift.  The ion's diffusivity field D(x) is carried in
// the electron-temperature component of the state: specDiff of the ion
// returns that component's value, so the implicit-diffusion solve sees a
// cell-by-cell coefficient field through the reference's own hook
// (specDiff(specid, Te, ndens, emag, Tg)) and harmonic face averaging.
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define ION_ID 1
#define NUM_SPECIES 2
#define NUM_IONS 1
#define FIRST_ION 1
#define NUM_NEUTRALS 0
#define FIRST_NEUTRAL 2
#define NUM_REACTIONS 0

inline void CKSYMS_STR(std::vector<std::string>& kname) { kname = {"E", "ION"}; }

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    return n == E_ID ? 0.000549 : 39.948;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[E_ID] = -1;
    kcharge[ION_ID] = 1;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return 0.0;
}

// the ion's diffusivity is the per-cell field held in the temperature slot
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specDiff(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return (specid == ION_ID) ? Te : 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const vd::Real T, vd::Real C[], vd::Real wdot[], const vd::Real Te, const vd::Real EN,
    vd::Real* ener_exch)
{
    for (int s = 0; s < NUM_SPECIES; ++s) wdot[s] = 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 0.0;
}
