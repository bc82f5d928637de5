"""Seeded plasma-chemistry mechanism generator.

Emits a case ``Chemistry.H`` with the hook set of the reference's generated
mechanisms (the CEPTR output shape of e.g. test/models/Streamer3d/Chemistry.H:
species table, CKCHRG, specMob/specDiff, productionRate + energy exchange by
reaction type, CKWC, etempLFA).  The reference generates these files from
Cantera YAML with py_utils/ceptr (Cantera is absent here); this generator
instead draws a charge-conserving mechanism from a seed, for the 8-species
LMEA benchmark configuration:

  species  E, P1..P4 (positive ions), NEG (negative ion), M (background
           gas, not transported), MX (transported excited neutral);
  rates    two-body  k = A Te^b exp(-Ea/Te), A log-uniform 1e-20..1e-14 m^3/s,
           b uniform -1..1, Ea uniform 0..15 eV (Te in eV);
           three-body A log-uniform 1e-44..1e-40 m^6/s;
  energy   electron energy exchange by reaction type (excitation/ionization
           loses Ea, recombination loses the mean electron energy) plus
           elastic collisions with the background, as comp_ener_exch in the
           reference's generated files.

Rates are evaluated as A exp(b ln Te - Ea/Te) with ln Te computed once per
cell (identical in exact arithmetic to A Te^b exp(-Ea/Te)).

  python -m vidyut_b200.mechgen --seed 2 --out vidyut_b200/cases/lmea8/Chemistry.H
"""
from __future__ import annotations

import argparse

import numpy as np

NA = 6.02214076e23
SPECIES = ["E", "P1", "P2", "P3", "P4", "NEG", "M", "MX"]
CHARGE = [-1, 1, 1, 1, 1, -1, 0, 0]
MW = [0.000549, 39.948, 28.014, 31.998, 44.01, 31.999, 39.948, 39.948]
E, POS, NEG, M, MX = 0, [1, 2, 3, 4], 5, 6, 7


def draw(seed: int, nreact: int = 30):
    rng = np.random.default_rng(seed)
    heavy_neutral = [M, MX]
    templates = ["ioniz", "excite", "deexcite", "recomb", "attach", "detach", "ionion",
                 "chargex", "penning", "threebody"]
    rx = []
    for r in range(nreact):
        t = templates[r % len(templates)] if r < len(templates) else templates[rng.integers(len(templates))]
        A = 10.0 ** rng.uniform(-20.0, -14.0)
        b = rng.uniform(-1.0, 1.0)
        Ea = rng.uniform(0.0, 15.0)
        p = POS[rng.integers(4)]
        p2 = POS[rng.integers(4)]
        m = heavy_neutral[rng.integers(2)]
        if t == "ioniz":        # E + m -> p + 2E
            reac, prod, typ = {E: 1, m: 1}, {p: 1, E: 2}, 2
        elif t == "excite":     # E + M -> E + MX
            reac, prod, typ = {E: 1, M: 1}, {E: 1, MX: 1}, 1
        elif t == "deexcite":   # E + MX -> E + M (superelastic: energy gain)
            reac, prod, typ = {E: 1, MX: 1}, {E: 1, M: 1}, 1
            Ea = -Ea  # energy returned to the electrons; no activation
        elif t == "recomb":     # E + p -> m
            reac, prod, typ, Ea = {E: 1, p: 1}, {m: 1}, 3, 0.0
        elif t == "attach":     # E + m -> NEG
            reac, prod, typ, Ea = {E: 1, m: 1}, {NEG: 1}, 4, 0.0
        elif t == "detach":     # NEG + m -> E + m
            reac, prod, typ, Ea = {NEG: 1, m: 1}, {E: 1, m: 1}, 7, 0.0
        elif t == "ionion":     # p + NEG -> 2 M
            reac, prod, typ, Ea = {p: 1, NEG: 1}, {M: 2}, 0, 0.0
        elif t == "chargex":    # p + m -> p2 + m
            if p2 == p:
                p2 = POS[(POS.index(p) + 1) % 4]
            reac, prod, typ, Ea = {p: 1, m: 1}, {p2: 1, m: 1}, 0, 0.0
        elif t == "penning":    # MX + MX -> p + E + M
            reac, prod, typ = {MX: 2}, {p: 1, E: 1, M: 1}, 6
            Ea = -Ea  # energy returned to the electrons; no activation
        else:                   # three-body: E + p + M -> m + M
            A = 10.0 ** rng.uniform(-44.0, -40.0)
            reac, prod, typ, Ea = {E: 1, p: 1, M: 1}, {m: 1, M: 1}, 3, 0.0
        q_r = sum(CHARGE[s] * n for s, n in reac.items())
        q_p = sum(CHARGE[s] * n for s, n in prod.items())
        assert q_r == q_p, (t, reac, prod)
        order = sum(reac.values())
        Amol = A * NA ** (order - 1)  # m^3/s -> m^3/mol/s (three-body: m^6/mol^2/s)
        rx.append(dict(t=t, reac=reac, prod=prod, typ=typ, A=Amol, b=b, Ea=Ea))
    return rx


def emit(seed: int) -> str:
    rx = draw(seed)
    L = []
    w = L.append
    w("// Generated by vidyut_b200/mechgen.py --seed %d; do not edit." % seed)
    w("// 8-species LMEA mechanism: E, P1..P4, NEG, M (background), MX.")
    w("#pragma once")
    w('#include "vd_defs.H"')
    w("#include <string>")
    w("#include <vector>")
    w("")
    for i, s in enumerate(SPECIES):
        w(f"#define {s}_ID {i}")
    w("#define NUM_SPECIES 8")
    w("#define NUM_IONS 5")
    w("#define FIRST_ION 1")
    w("#define NUM_NEUTRALS 2")
    w("#define FIRST_NEUTRAL 6")
    w(f"#define NUM_REACTIONS {len(rx)}")
    w("#define LMEA_SEED %d" % seed)
    w("")
    w("inline void CKSYMS_STR(std::vector<std::string>& kname)")
    w("{")
    w("    kname = {" + ", ".join(f'"{s}"' for s in SPECIES) + "};")
    w("}")
    w("")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE vd::Real mw(const int n)")
    w("{")
    w("    const vd::Real w[8] = {" + ", ".join(repr(x) for x in MW) + "};")
    w("    return w[n];")
    w("}")
    w("")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void CKCHRG(int kcharge[])")
    w("{")
    for i, q in enumerate(CHARGE):
        w(f"    kcharge[{i}] = {q};")
    w("}")
    w("")
    w("""// Mobilities from collision frequencies with the gas (cross sections
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
""")
    w("""// Reaction rates q_r (mol/m^3/s) from concentrations C (mol/m^3) at the
// electron temperature Te (K); th (may be null) shifts the log pre-factors.
template <class R>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_rates(
    const vd::Real T, const R* C, const vd::Real Te, const vd::Real* th, R* q)
{
    const vd::Real TeV = Te / eV;
    const vd::Real lnTe = std::log(TeV);
    const vd::Real iTe = 1.0 / TeV;""")
    for r, d in enumerate(rx):
        conc = " * ".join(f"C[{s}]" + (f" * C[{s}]" if n == 2 else "") for s, n in d["reac"].items())
        ea_rate = max(d["Ea"], 0.0)
        w(f"    q[{r}] = {d['A']!r} * std::exp({d['b']!r} * lnTe - {ea_rate!r} * iTe + "
          f"(th ? th[{r}] : 0.0)) * {conc};")
    w("}")
    w("")
    w("// Net production rates from reaction rates (stoichiometry).")
    w("template <class R>")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_wdot(const R* q, R* wdot)")
    w("{")
    w("    for (int i = 0; i < NUM_SPECIES; ++i) wdot[i] = R(0.0);")
    nets = []
    for r, d in enumerate(rx):
        net = {}
        for s_, n in d["reac"].items():
            net[s_] = net.get(s_, 0) - n
        for s_, n in d["prod"].items():
            net[s_] = net.get(s_, 0) + n
        nets.append(net)
        for s_, n in sorted(net.items()):
            if n:
                w(f"    wdot[{s_}] += {float(n)!r} * q[{r}];")
    w("}")
    w("")
    w("// out[r] = sum_s nu[s][r] lam[s]: the stoichiometry transposed onto lam.")
    w("AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void mech_lam_nu(const vd::Real* lam, vd::Real* out)")
    w("{")
    for r, net in enumerate(nets):
        terms = " + ".join(f"{float(n)!r} * lam[{s_}]" for s_, n in sorted(net.items()) if n)
        w(f"    out[{r}] = {terms or '0.0'};")
    w("}")
    w("")
    w("#define VD_HAS_MECH_ADJOINT 1")
    w("")
    w("""// Molar production rates (mol/m^3/s) and electron energy exchange (W/m^3)
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
    const vd::Real sefact = (std::tanh((Te - T) / 0.5) + 1.0) / 2.0;""")
    for r, d in enumerate(rx):
        if d["typ"] in (1, 2, 6) and d["Ea"] != 0.0:
            w(f"    *ener_exch -= ({d['Ea']!r} * eV2J) * N_A * q[{r}] * sefact;")
        elif d["typ"] == 3:
            w(f"    *ener_exch -= mee * N_A * q[{r}];")
    w("""    // elastic electron-gas collisions
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
}""")
    return "\n".join(L) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    with open(a.out, "w") as f:
        f.write(emit(a.seed))


if __name__ == "__main__":
    main()
