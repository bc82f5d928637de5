// Method-of-manufactured-solutions case 3 of the reference
// (test/verification/MMS3): time accuracy of the step.  No transport (all
// mobilities and diffusivities zero); per cell
//   dn_e/dt = dn_i/dt = k_i n_e with k_i = -5 (the reaction HE + E with a
//   negative rate constant and the background neutral HE at 1 m^-3),
//   dE_eps/dt = -10 E_eps (a user source),
// so from n0 (1 + sin(pi x / L)) the exact solution decays as exp(-5 t)
// and exp(-10 t) (test/verification/MMS3/README.md, l2err/l2err.cpp:
// 100-134).  The reaction's energy exchange and elastic loss are zero
// (zero excitation energy, zero collision frequency).
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define HE_ID 1
#define HEp_ID 2
#define NUM_SPECIES 3
#define NUM_IONS 1
#define FIRST_ION 2
#define NUM_NEUTRALS 1
#define FIRST_NEUTRAL 1
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

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return 0.0;
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
    for (int s = 0; s < NUM_SPECIES; ++s) wdot[s] = 0.0;
    *ener_exch = 0.0;
    const vd::Real kf = -5.0 * 6.02214076e23;
    const vd::Real q = kf * (C[E_ID] * C[HE_ID]);
    wdot[E_ID] += q;
    wdot[HE_ID] -= q;
    wdot[HEp_ID] += q;
    // ionization with zero excitation energy, superelastic factor as the
    // reference's energy-exchange routine forms it
    const vd::Real ev2j = 1.602176620800000e-19;
    const vd::Real se = (std::tanh((Te - T) / 0.5) + 1.0) / 2.0;
    *ener_exch -= (0.0 * ev2j) * 6.02214085774e23 * q * se;
    // elastic loss at zero collision frequency
    const vd::Real nu = 0.0;
    *ener_exch -= 3.0 / 2.0 * C[E_ID] * N_A * (K_B * Te - K_B * T) * nu * (2.0 * ME / (4.0 * M_AMU));
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 5802.25;
}
