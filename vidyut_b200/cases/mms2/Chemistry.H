// Method-of-manufactured-solutions case 2 of the reference
// (test/verification/MMS2): the full drift-diffusion model with the
// electron-energy equation.  Species: electrons E, a background neutral HE
// and one ion HEp; one ionization reaction HE + E -> HEp + 2E with
//   k_i = 5 exp(-Ta/Te) (times N_A in mol units), Ta = 2/kB,
// an inelastic loss of 4 J per ionization and elastic losses at
// nu = 1e4 /s with m_h = 4 amu (test/verification/MMS2/Chemistry.H:250-330).
// Transport: mu_e = -1, D_e = 1, mu_i = 0.5, D_i = 0.5 (energy: 5/3 of the
// electron values).  Exact steady solution along the axial direction x:
//   n_e = x^3/alpha + n0, n_i = x^3/(2 alpha) + n0, E_eps = n_e,
//   phi = (x^5 - x)/40, alpha = e/eps0, n0 = 1e6
// (test/verification/MMS2/UserSources.H:50-100, l2err/l2err.cpp:176-194).
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define HE_ID 1
#define HEp_ID 2
#define NUM_SPECIES 3
#define FIRST_ION 2
#define NUM_IONS 1
#define FIRST_NEUTRAL 0
#define NUM_NEUTRALS 0
#define NUM_REACTIONS 1

inline void CKSYMS_STR(std::vector<std::string>& kname) { kname = {"E", "HE", "HEp"}; }

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    return n == E_ID ? 0.000549 : 4.002602;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[E_ID] = -1;
    kcharge[HE_ID] = 0;
    kcharge[HEp_ID] = 1;
}

// charge-signed mobility; specid == NUM_SPECIES is the electron energy
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    if (specid == E_ID) return -1.0;
    if (specid == HEp_ID) return 0.5;
    if (specid == NUM_SPECIES) return fivebythree * -1.0;
    return 0.0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specDiff(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    if (specid == E_ID) return 1.0;
    if (specid == HEp_ID) return 0.5;
    if (specid == NUM_SPECIES) return fivebythree * 1.0;
    return 0.0;
}

// Production rates (mol/m^3/s) and electron-energy exchange (J/m^3/s) of
// the single ionization reaction, with the reference's constants.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const vd::Real T, vd::Real C[], vd::Real wdot[], const vd::Real Te, const vd::Real EN,
    vd::Real* ener_exch)
{
    const vd::Real na_rate = 6.02214076e23;   // N_A of the rate constant
    const vd::Real na = 6.02214085774e23;     // N_A of the energy terms
    const vd::Real ev2j = 1.602176620800000e-19;
    for (int s = 0; s < NUM_SPECIES; ++s) wdot[s] = 0.0;
    *ener_exch = 0.0;
    const vd::Real Ta = 2.0 / K_B;
    const vd::Real kf = 5.0 * std::exp(-Ta / Te) * na_rate;
    const vd::Real q = kf * (C[E_ID] * C[HE_ID]);
    wdot[E_ID] += q;
    wdot[HE_ID] -= q;
    wdot[HEp_ID] += q;
    // ionization energy 4/ev2j eV per event, scaled by the superelastic factor
    const vd::Real se = (std::tanh((Te - T) / 0.5) + 1.0) / 2.0;
    *ener_exch -= ((4.0 / ev2j) * ev2j) * na * q * se;
    // elastic collisions with the 4-amu heavies at nu = 1e4 /s
    const vd::Real nu = 10000.0;
    *ener_exch -= 3.0 / 2.0 * C[E_ID] * N_A * (K_B * Te - K_B * T) * nu * (2.0 * ME / (4.0 * M_AMU));
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 5802.25;
}
