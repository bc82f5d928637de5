// Generated by vidyut_b200/mechgen.py --seed 2; do not edit.
// 8-species LMEA mechanism: E, P1..P4, NEG, M (background), MX.
#pragma once
#include "vd_defs.H"
#include <string>
#include <vector>

#define E_ID 0
#define P1_ID 1
#define P2_ID 2
#define P3_ID 3
#define P4_ID 4
#define NEG_ID 5
#define M_ID 6
#define MX_ID 7
#define NUM_SPECIES 8
#define NUM_IONS 5
#define FIRST_ION 1
#define NUM_NEUTRALS 2
#define FIRST_NEUTRAL 6
#define NUM_REACTIONS 30
#define LMEA_SEED 2

inline void CKSYMS_STR(std::vector<std::string>& kname)
{
    kname = {"E", "P1", "P2", "P3", "P4", "NEG", "M", "MX"};
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)
{
    const vd::Real w[8] = {0.000549, 39.948, 28.014, 31.998, 44.01, 31.999, 39.948, 39.948};
    return w[n];
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])
{
    kcharge[0] = -1;
    kcharge[1] = 1;
    kcharge[2] = 1;
    kcharge[3] = 1;
    kcharge[4] = 1;
    kcharge[5] = -1;
    kcharge[6] = 0;
    kcharge[7] = 0;
}

// Mobilities from collision frequencies with the gas (cross sections
// 40e-20 m^2 for electrons, 120e-20 m^2 for heavies), charge-signed; the
// electron energy uses 5/3 of the electron values.  Templated on the number
// type so the adjoint can differentiate them with respect to the density.
template <class R>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE R specMob_T(
    const int specid, const R& Te, const R& ndens, const R& emag, const vd::Real T)
{
    using std::sqrt;
    const R nu_e = sqrt(8.0 * K_B * Te / PI / ME) * ndens * 40e-20;
    const R elecmob = -ECHARGE / ME / nu_e;
    if (specid == E_ID) return elecmob;
    if (specid == NUM_SPECIES) return fivebythree * elecmob;
    const int q[8] = {-1, 1, 1, 1, 1, -1, 0, 0};
    if (specid < 0 || specid >= NUM_SPECIES || q[specid] == 0) return R(0.0);
    const vd::Real m = mw(specid) * M_AMU;
    const R nu = std::sqrt(8.0 * K_B * T / PI / m) * ndens * 120e-20;
    return q[specid] * ECHARGE / m / nu;
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specMob(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    return specMob_T<vd::Real>(specid, Te, ndens, emag, T);
}

AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real specDiff(
    const int specid, const vd::Real Te, const vd::Real ndens, const vd::Real emag,
    const vd::Real T)
{
    const vd::Real elecmob = specMob(E_ID, Te, ndens, emag, T);
    if (specid == E_ID) return Te / eV * std::fabs(elecmob);
    if (specid == NUM_SPECIES) return fivebythree * Te / eV * std::fabs(elecmob);
    const vd::Real m = (specid >= 0 && specid < NUM_SPECIES) ? mw(specid) * M_AMU : M_AMU;
    const vd::Real nu = std::sqrt(8.0 * K_B * T / PI / m) * ndens * 120e-20;
    return T / eV * ECHARGE / m / nu;
}

// Reaction rates q_r (mol/m^3/s) from concentrations C (mol/m^3) at the
// electron temperature Te (K); th (may be null) shifts the log pre-factors.
template <class R>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_rates(
    const vd::Real T, const R* C, const vd::Real Te, const vd::Real* th, R* q)
{
    const vd::Real TeV = Te / eV;
    const vd::Real lnTe = std::log(TeV);
    const vd::Real iTe = 1.0 / TeV;
    q[0] = 223575.24116184682 * std::exp(-0.4030177131717534 * lnTe - 12.213386108914206 * iTe + (th ? th[0] : 0.0)) * C[0] * C[6];
    q[1] = 141616567.33697075 * std::exp(-0.6241978532667931 * lnTe - 0.8271994099960228 * iTe + (th ? th[1] : 0.0)) * C[0] * C[6];
    q[2] = 53008924.346136846 * std::exp(0.124531325560856 * lnTe - 0.0 * iTe + (th ? th[2] : 0.0)) * C[0] * C[7];
    q[3] = 2072330.1332144644 * std::exp(0.2663687985482328 * lnTe - 0.0 * iTe + (th ? th[3] : 0.0)) * C[0] * C[3];
    q[4] = 1347410.4177761925 * std::exp(-0.6254948605598039 * lnTe - 0.0 * iTe + (th ? th[4] : 0.0)) * C[0] * C[7];
    q[5] = 271103145.91733485 * std::exp(-0.36370679876925127 * lnTe - 0.0 * iTe + (th ? th[5] : 0.0)) * C[5] * C[6];
    q[6] = 87559637.63980156 * std::exp(-0.7855853830928239 * lnTe - 0.0 * iTe + (th ? th[6] : 0.0)) * C[4] * C[5];
    q[7] = 72213712.2815985 * std::exp(0.6984726472288691 * lnTe - 0.0 * iTe + (th ? th[7] : 0.0)) * C[4] * C[6];
    q[8] = 7572164.97068507 * std::exp(0.1868870355118124 * lnTe - 0.0 * iTe + (th ? th[8] : 0.0)) * C[7] * C[7];
    q[9] = 82338.5668092122 * std::exp(0.6587122516131629 * lnTe - 0.0 * iTe + (th ? th[9] : 0.0)) * C[0] * C[4] * C[6];
    q[10] = 119423.89965973822 * std::exp(-0.7985927959630463 * lnTe - 0.0 * iTe + (th ? th[10] : 0.0)) * C[3] * C[7];
    q[11] = 1466073639.121359 * std::exp(0.6703664093845594 * lnTe - 0.0 * iTe + (th ? th[11] : 0.0)) * C[5] * C[7];
    q[12] = 237165103.7308681 * std::exp(-0.1856112830407861 * lnTe - 0.0 * iTe + (th ? th[12] : 0.0)) * C[3] * C[6];
    q[13] = 25268764.387723103 * std::exp(-0.7747342897773635 * lnTe - 0.0 * iTe + (th ? th[13] : 0.0)) * C[0] * C[7];
    q[14] = 3042692.8622457315 * std::exp(-0.023002853832061243 * lnTe - 0.0 * iTe + (th ? th[14] : 0.0)) * C[0] * C[1];
    q[15] = 191483108.25504968 * std::exp(0.14893299576593155 * lnTe - 0.0 * iTe + (th ? th[15] : 0.0)) * C[0] * C[7];
    q[16] = 137881.907373414 * std::exp(0.37805427429713667 * lnTe - 0.0 * iTe + (th ? th[16] : 0.0)) * C[5] * C[6];
    q[17] = 2201671470.370027 * std::exp(0.5691297148599996 * lnTe - 0.0 * iTe + (th ? th[17] : 0.0)) * C[2] * C[6];
    q[18] = 555331821.7846208 * std::exp(-0.779264815381874 * lnTe - 0.0 * iTe + (th ? th[18] : 0.0)) * C[0] * C[7];
    q[19] = 489901.6439024877 * std::exp(-0.9019732208738158 * lnTe - 0.0 * iTe + (th ? th[19] : 0.0)) * C[0] * C[2];
    q[20] = 6613.992548252871 * std::exp(-0.7040742394195629 * lnTe - 0.0 * iTe + (th ? th[20] : 0.0)) * C[3] * C[6];
    q[21] = 28821525.326525826 * std::exp(-0.4291347889214092 * lnTe - 0.0 * iTe + (th ? th[21] : 0.0)) * C[2] * C[7];
    q[22] = 108170.5946844993 * std::exp(0.12604636651181567 * lnTe - 0.0 * iTe + (th ? th[22] : 0.0)) * C[0] * C[7];
    q[23] = 3311857.427522815 * std::exp(0.3373815171003467 * lnTe - 0.0 * iTe + (th ? th[23] : 0.0)) * C[7] * C[7];
    q[24] = 12477.964986217788 * std::exp(0.953272986584375 * lnTe - 0.0 * iTe + (th ? th[24] : 0.0)) * C[0] * C[7];
    q[25] = 31935624.249445166 * std::exp(-0.22871976623272094 * lnTe - 6.699052132358132 * iTe + (th ? th[25] : 0.0)) * C[0] * C[6];
    q[26] = 11494042.09859202 * std::exp(0.5849022081088895 * lnTe - 0.0 * iTe + (th ? th[26] : 0.0)) * C[7] * C[7];
    q[27] = 3854240392.478695 * std::exp(-0.9120246158872058 * lnTe - 0.0 * iTe + (th ? th[27] : 0.0)) * C[0] * C[3];
    q[28] = 86162.98868308256 * std::exp(0.09738275198198632 * lnTe - 4.339168861828789 * iTe + (th ? th[28] : 0.0)) * C[0] * C[6];
    q[29] = 1662612424.3660362 * std::exp(0.34180863007165474 * lnTe - 0.0 * iTe + (th ? th[29] : 0.0)) * C[5] * C[6];
}

// Net production rates from reaction rates (stoichiometry).
template <class R>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_wdot(const R* q, R* wdot)
{
    for (int i = 0; i < NUM_SPECIES; ++i) wdot[i] = R(0.0);
    wdot[0] += 1.0 * q[0];
    wdot[2] += 1.0 * q[0];
    wdot[6] += -1.0 * q[0];
    wdot[6] += -1.0 * q[1];
    wdot[7] += 1.0 * q[1];
    wdot[6] += 1.0 * q[2];
    wdot[7] += -1.0 * q[2];
    wdot[0] += -1.0 * q[3];
    wdot[3] += -1.0 * q[3];
    wdot[7] += 1.0 * q[3];
    wdot[0] += -1.0 * q[4];
    wdot[5] += 1.0 * q[4];
    wdot[7] += -1.0 * q[4];
    wdot[0] += 1.0 * q[5];
    wdot[5] += -1.0 * q[5];
    wdot[4] += -1.0 * q[6];
    wdot[5] += -1.0 * q[6];
    wdot[6] += 2.0 * q[6];
    wdot[2] += 1.0 * q[7];
    wdot[4] += -1.0 * q[7];
    wdot[0] += 1.0 * q[8];
    wdot[1] += 1.0 * q[8];
    wdot[6] += 1.0 * q[8];
    wdot[7] += -2.0 * q[8];
    wdot[0] += -1.0 * q[9];
    wdot[4] += -1.0 * q[9];
    wdot[7] += 1.0 * q[9];
    wdot[3] += -1.0 * q[10];
    wdot[4] += 1.0 * q[10];
    wdot[0] += 1.0 * q[11];
    wdot[5] += -1.0 * q[11];
    wdot[3] += -1.0 * q[12];
    wdot[4] += 1.0 * q[12];
    wdot[0] += -1.0 * q[13];
    wdot[5] += 1.0 * q[13];
    wdot[7] += -1.0 * q[13];
    wdot[0] += -1.0 * q[14];
    wdot[1] += -1.0 * q[14];
    wdot[7] += 1.0 * q[14];
    wdot[0] += -1.0 * q[15];
    wdot[5] += 1.0 * q[15];
    wdot[7] += -1.0 * q[15];
    wdot[0] += 1.0 * q[16];
    wdot[5] += -1.0 * q[16];
    wdot[1] += 1.0 * q[17];
    wdot[2] += -1.0 * q[17];
    wdot[0] += -1.0 * q[18];
    wdot[5] += 1.0 * q[18];
    wdot[7] += -1.0 * q[18];
    wdot[0] += -1.0 * q[19];
    wdot[2] += -1.0 * q[19];
    wdot[6] += 1.0 * q[19];
    wdot[3] += -1.0 * q[20];
    wdot[4] += 1.0 * q[20];
    wdot[2] += -1.0 * q[21];
    wdot[3] += 1.0 * q[21];
    wdot[6] += 1.0 * q[22];
    wdot[7] += -1.0 * q[22];
    wdot[0] += 1.0 * q[23];
    wdot[1] += 1.0 * q[23];
    wdot[6] += 1.0 * q[23];
    wdot[7] += -2.0 * q[23];
    wdot[6] += 1.0 * q[24];
    wdot[7] += -1.0 * q[24];
    wdot[6] += -1.0 * q[25];
    wdot[7] += 1.0 * q[25];
    wdot[0] += 1.0 * q[26];
    wdot[4] += 1.0 * q[26];
    wdot[6] += 1.0 * q[26];
    wdot[7] += -2.0 * q[26];
    wdot[0] += -1.0 * q[27];
    wdot[3] += -1.0 * q[27];
    wdot[7] += 1.0 * q[27];
    wdot[6] += -1.0 * q[28];
    wdot[7] += 1.0 * q[28];
    wdot[0] += 1.0 * q[29];
    wdot[5] += -1.0 * q[29];
}

// out[r] = sum_s nu[s][r] lam[s]: the stoichiometry transposed onto lam.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_lam_nu(const vd::Real* lam, vd::Real* out)
{
    out[0] = 1.0 * lam[0] + 1.0 * lam[2] + -1.0 * lam[6];
    out[1] = -1.0 * lam[6] + 1.0 * lam[7];
    out[2] = 1.0 * lam[6] + -1.0 * lam[7];
    out[3] = -1.0 * lam[0] + -1.0 * lam[3] + 1.0 * lam[7];
    out[4] = -1.0 * lam[0] + 1.0 * lam[5] + -1.0 * lam[7];
    out[5] = 1.0 * lam[0] + -1.0 * lam[5];
    out[6] = -1.0 * lam[4] + -1.0 * lam[5] + 2.0 * lam[6];
    out[7] = 1.0 * lam[2] + -1.0 * lam[4];
    out[8] = 1.0 * lam[0] + 1.0 * lam[1] + 1.0 * lam[6] + -2.0 * lam[7];
    out[9] = -1.0 * lam[0] + -1.0 * lam[4] + 1.0 * lam[7];
    out[10] = -1.0 * lam[3] + 1.0 * lam[4];
    out[11] = 1.0 * lam[0] + -1.0 * lam[5];
    out[12] = -1.0 * lam[3] + 1.0 * lam[4];
    out[13] = -1.0 * lam[0] + 1.0 * lam[5] + -1.0 * lam[7];
    out[14] = -1.0 * lam[0] + -1.0 * lam[1] + 1.0 * lam[7];
    out[15] = -1.0 * lam[0] + 1.0 * lam[5] + -1.0 * lam[7];
    out[16] = 1.0 * lam[0] + -1.0 * lam[5];
    out[17] = 1.0 * lam[1] + -1.0 * lam[2];
    out[18] = -1.0 * lam[0] + 1.0 * lam[5] + -1.0 * lam[7];
    out[19] = -1.0 * lam[0] + -1.0 * lam[2] + 1.0 * lam[6];
    out[20] = -1.0 * lam[3] + 1.0 * lam[4];
    out[21] = -1.0 * lam[2] + 1.0 * lam[3];
    out[22] = 1.0 * lam[6] + -1.0 * lam[7];
    out[23] = 1.0 * lam[0] + 1.0 * lam[1] + 1.0 * lam[6] + -2.0 * lam[7];
    out[24] = 1.0 * lam[6] + -1.0 * lam[7];
    out[25] = -1.0 * lam[6] + 1.0 * lam[7];
    out[26] = 1.0 * lam[0] + 1.0 * lam[4] + 1.0 * lam[6] + -2.0 * lam[7];
    out[27] = -1.0 * lam[0] + -1.0 * lam[3] + 1.0 * lam[7];
    out[28] = -1.0 * lam[6] + 1.0 * lam[7];
    out[29] = 1.0 * lam[0] + -1.0 * lam[5];
}

#define VD_HAS_MECH_ADJOINT 1

// Molar production rates (mol/m^3/s) and electron energy exchange (W/m^3)
// from concentrations C (mol/m^3), gas and electron temperatures (K).
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKWC(
    const vd::Real T, vd::Real C[], vd::Real wdot[], const vd::Real Te, const vd::Real EN,
    vd::Real* ener_exch)
{
    vd::Real q[NUM_REACTIONS];
    mech_rates<vd::Real>(T, C, Te, nullptr, q);
    mech_wdot<vd::Real>(q, wdot);
    const vd::Real eV2J = ECHARGE;
    const vd::Real ne = C[E_ID] * N_A;
    const vd::Real mee = (ne > 0.0) ? 1.5 * K_B * Te : 0.0; // mean electron energy (J)
    const vd::Real sefact = (std::tanh((Te - T) / 0.5) + 1.0) / 2.0;
    *ener_exch -= (12.213386108914206 * eV2J) * N_A * q[0] * sefact;
    *ener_exch -= (0.8271994099960228 * eV2J) * N_A * q[1] * sefact;
    *ener_exch -= (-2.250933949580042 * eV2J) * N_A * q[2] * sefact;
    *ener_exch -= mee * N_A * q[3];
    *ener_exch -= (-12.931769773614421 * eV2J) * N_A * q[8] * sefact;
    *ener_exch -= mee * N_A * q[9];
    *ener_exch -= mee * N_A * q[14];
    *ener_exch -= mee * N_A * q[19];
    *ener_exch -= (-11.559903442259692 * eV2J) * N_A * q[22] * sefact;
    *ener_exch -= (-13.549918904832174 * eV2J) * N_A * q[23] * sefact;
    *ener_exch -= (-9.219419237267353 * eV2J) * N_A * q[24] * sefact;
    *ener_exch -= (6.699052132358132 * eV2J) * N_A * q[25] * sefact;
    *ener_exch -= (-6.090073936395816 * eV2J) * N_A * q[26] * sefact;
    *ener_exch -= mee * N_A * q[27];
    *ener_exch -= (4.339168861828789 * eV2J) * N_A * q[28] * sefact;
    // elastic electron-gas collisions
    vd::Real nd = 0.0;
    for (int sp = 0; sp < NUM_SPECIES; sp++) nd += C[sp] * N_A;
    const vd::Real mu = specMob(E_ID, Te, nd, 0.0, T);
    const vd::Real nu = -ECHARGE / ME / mu;
    *ener_exch -= 1.5 * K_B * C[E_ID] * N_A * (Te - T) * nu * (2.0 * ME / (39.948 * M_AMU));
}

// Local-field electron temperature: 1 eV.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real
etempLFA(const vd::Real Tg, vd::Real C[], const vd::Real EN)
{
    return 11604.518;
}
