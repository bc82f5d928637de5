// Two-species Townsend discharge (electrons + one positive ion) in a
// background gas held as a third, non-transported species.  Hook names and
// signatures follow the reference's case Chemistry.H (e.g.
// test/verification/Streamer_Axisym/Chemistry.H:180-292).
//
// Coefficients: electron mobility 0.0382 m^2/Vs (charge-signed, so -0.0382),
// electron diffusion 0.18 m^2/s; ion mobility 2e-4 m^2/Vs, ion diffusion
// 5e-6 m^2/s.  Ionization by Townsend alpha = A p exp(-B p / |E|) with
// A = 1.2e3 /(m Torr), B = 3.42e4 V/(m Torr), p = 760 Torr, so that the
// electron and ion sources are alpha |mu_e| |E| n_e.
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define ION_ID 1
#define N_ID 2
#define NUM_SPECIES 3
#define NUM_IONS 1
#define FIRST_ION 1
#define NUM_NEUTRALS 0
#define FIRST_NEUTRAL 2
#define NUM_REACTIONS 1

#define TOWNSEND_MU_E 0.0382
#define TOWNSEND_D_E 0.18
#define TOWNSEND_MU_I 2.0e-4
#define TOWNSEND_D_I 5.0e-6
#define TOWNSEND_A 1.2e3
#define TOWNSEND_B 3.42e4
#define TOWNSEND_P_TORR 760.0

inline void CKSYMS_STR(std::vector<std::string>& kname)
{
    kname = {"E", "ION", "N"};
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    const vd::Real w[3] = {0.000549, 28.014, 28.014};
    return w[n];
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[0] = -1;
    kcharge[1] = 1;
    kcharge[2] = 0;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens,
    const vd::Real emag, const vd::Real T)
{
    vd::Real mob = 0.0;
    if (specid == E_ID) mob = -TOWNSEND_MU_E;
    if (specid == ION_ID) mob = TOWNSEND_MU_I;
    if (specid == NUM_SPECIES) mob = (5.0 / 3.0) * (-TOWNSEND_MU_E);
    return mob;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specDiff(
    const int specid, const vd::Real Te, const vd::Real ndens,
    const vd::Real emag, const vd::Real T)
{
    vd::Real d = 0.0;
    if (specid == E_ID) d = TOWNSEND_D_E;
    if (specid == ION_ID) d = TOWNSEND_D_I;
    if (specid == NUM_SPECIES) d = (5.0 / 3.0) * TOWNSEND_D_E;
    return d;
}

// Molar production rates (mol/m^3/s) from concentrations C (mol/m^3).
// |E| is recovered from the reduced field EN (Td) with the heavy-particle
// density sum(C) - C_e, the same denominator the field solve uses
// (Source/PotentialSolve.cpp:526-534).
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const vd::Real T, vd::Real C[], vd::Real wdot[], const vd::Real Te,
    const vd::Real EN, vd::Real* ener_exch)
{
    for (int i = 0; i < NUM_SPECIES; ++i) wdot[i] = 0.0;
    const vd::Real nheavy = (C[ION_ID] + C[N_ID]) * N_A;
    const vd::Real emag = vd::vmax(1e-10, EN * nheavy * 1.0e-21);
    const vd::Real alpha = TOWNSEND_A * TOWNSEND_P_TORR *
                           std::exp(-TOWNSEND_B * TOWNSEND_P_TORR / emag);
    const vd::Real k_f = alpha * TOWNSEND_MU_E * emag;
    wdot[E_ID] += k_f * C[E_ID];
    wdot[ION_ID] += k_f * C[E_ID];
}

// Local-field electron temperature: fixed at 0.5 eV.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 5802.25;
}
