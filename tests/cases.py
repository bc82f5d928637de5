"""Inputs of the verification cases shared by the oracle and GPU tests,
written as reference inputs-file text (ParmParse names)."""
from __future__ import annotations

import numpy as np

import vidyut_b200 as vb


def mms1_config(n: int, hyp: int = 5, dt: float = 0.1) -> vb.Config:
    # test/verification/MMS1/inputs_x with amr.max_level=0 (single level)
    txt = f"""
amr.n_cell = {n} 4 4
geometry.prob_hi = 1.0 0.125 0.125
geometry.is_periodic = 0 1 1
vidyut.dt = {dt}
vidyut.hyp_order = {hyp}
vidyut.user_defined_potential = 1
vidyut.user_defined_species = 1
vidyut.user_defined_vel = 1
vidyut.pot_bc_lo = 4 0 0
vidyut.pot_bc_hi = 4 0 0
vidyut.eden_bc_lo = 2 0 0
vidyut.eden_bc_hi = 2 0 0
vidyut.ion_bc_lo = 4 0 0
vidyut.ion_bc_hi = 4 0 0
"""
    return vb.Config.from_inputs("mms1", txt)


def mms1_errors(S: np.ndarray, n: int) -> tuple[float, float]:
    info = vb.case_info("mms1")
    x = (np.arange(n) + 0.5) / n
    ni = S[1].mean(axis=(0, 1))
    pot = S[info["pot_id"]].mean(axis=(0, 1))
    return (float(np.sqrt(np.mean((ni - x ** 2) ** 2))),
            float(np.sqrt(np.mean((pot - (x ** 4 - x) / 12) ** 2))))


def advect_config(n: int, dt: float = 2.5e-4, weno: int = 3) -> vb.Config:
    # test/verification/Advect/inputs1d: 2-D, periodic, WENO5, two correctors
    cfg = vb.Config("advect")
    cfg["dim"] = 2
    cfg.set("amr.n_cell", f"{n} 4 1")
    cfg.set("geometry.prob_lo", "-1 0 0")
    cfg.set("geometry.prob_hi", "1 0.4 1")
    cfg.set("geometry.is_periodic", "1 1 0")
    cfg["dt"] = dt
    cfg["hyp_order"] = 5
    cfg["weno_scheme"] = weno
    cfg["num_timestep_correctors"] = 2
    cfg["user_defined_potential"] = 1
    cfg["user_defined_species"] = 1
    cfg["user_defined_vel"] = 1
    for key in ("pot", "eden", "ion", "neutral", "eenrg"):
        cfg[f"{key}_bc_lo"] = [0, 0, 0]
        cfg[f"{key}_bc_hi"] = [0, 0, 0]
    return cfg


ADVECT_PROB = "prob.one_dim = 1\nprob.velx = 1.0"


def advect_error(S: np.ndarray, n: int, T: float) -> float:
    x = -1 + (np.arange(n) + 0.5) * 2.0 / n
    ex = np.sin(np.pi * (x - T) - np.sin(np.pi * (x - T)) / np.pi)
    return float(np.sqrt(np.mean((S[1, 0, 2] - ex) ** 2)))


def mms2_config(n: int, hyp: int = 5, dt: float = 0.05, ny: int = 4) -> vb.Config:
    # test/verification/MMS2/inputs_x with amr.max_level=0 (single level)
    txt = f"""
amr.n_cell = {n} {ny} {ny}
geometry.prob_hi = 1.0 0.125 0.125
geometry.is_periodic = 0 1 1
vidyut.dt = {dt}
vidyut.hyp_order = {hyp}
vidyut.user_defined_potential = 1
vidyut.user_defined_species = 1
vidyut.user_defined_vel = 1
vidyut.bound_specden = 1
vidyut.min_species_density = 1e-11
vidyut.min_electron_density = 1e-11
vidyut.min_electron_temp = 1e-11
vidyut.linsolve_maxiter = 200
vidyut.elecenergy_solve = 1
vidyut.bg_species_ids = 1
vidyut.gas_temperature = 1e-50
vidyut.pot_bc_lo = 4 0 0
vidyut.pot_bc_hi = 4 0 0
vidyut.eden_bc_lo = 1 0 0
vidyut.eden_bc_hi = 1 0 0
vidyut.eenrg_bc_lo = 1 0 0
vidyut.eenrg_bc_hi = 1 0 0
vidyut.ion_bc_lo = 1 0 0
vidyut.ion_bc_hi = 1 0 0
vidyut.neutral_bc_lo = 2 0 0
vidyut.neutral_bc_hi = 2 0 0
"""
    return vb.Config.from_inputs("mms2", txt)


MMS2_ALPHA = 1.60217662e-19 / 8.854187817e-12
MMS2_N0 = 1e6


def mms2_errors(S: np.ndarray, n: int) -> tuple[float, float]:
    """The reference's l2err metric (test/verification/MMS2/l2err/
    l2err.cpp:176-194): RMS error over the domain divided by the domain
    average, for the electron density and the potential."""
    info = vb.case_info("mms2")
    x = (np.arange(n) + 0.5) / n
    ne = S[0]
    pot = S[info["pot_id"]]
    ex_ne = x ** 3 / MMS2_ALPHA + MMS2_N0
    ex_pot = (x ** 5 - x) / 40.0
    err_e = np.sqrt(np.mean((ne - ex_ne) ** 2)) / np.mean(ne)
    err_p = np.sqrt(np.mean((pot - ex_pot) ** 2)) / abs(np.mean(pot))
    return float(err_e), float(err_p)


def mms3_config(dt: float, correctors: int, n: int = 16) -> vb.Config:
    # test/verification/MMS3/inputs with run1.sh / run2.sh's dt and
    # corrector counts (amr.max_level = 0 in the reference's inputs)
    txt = f"""
amr.n_cell = {n} 4 4
geometry.prob_hi = 1.0 0.125 0.125
geometry.is_periodic = 0 1 1
vidyut.dt = {dt}
vidyut.num_timestep_correctors = {correctors}
vidyut.user_defined_potential = 1
vidyut.user_defined_species = 1
vidyut.user_defined_vel = 1
vidyut.bound_specden = 1
vidyut.min_species_density = 1e-11
vidyut.min_electron_density = 1e-11
vidyut.min_electron_temp = 1e-11
vidyut.linsolve_maxiter = 200
vidyut.elecenergy_solve = 1
vidyut.bg_species_ids = 1
vidyut.gas_temperature = 1e-50
vidyut.pot_bc_lo = 2 0 0
vidyut.pot_bc_hi = 2 0 0
vidyut.eden_bc_lo = 2 0 0
vidyut.eden_bc_hi = 2 0 0
vidyut.eenrg_bc_lo = 2 0 0
vidyut.eenrg_bc_hi = 2 0 0
vidyut.ion_bc_lo = 2 0 0
vidyut.ion_bc_hi = 2 0 0
vidyut.neutral_bc_lo = 2 0 0
vidyut.neutral_bc_hi = 2 0 0
"""
    return vb.Config.from_inputs("mms3", txt)


def mms3_errors(S: np.ndarray, n: int, t: float) -> tuple[float, float]:
    """Relative L2 errors of the electron density and the electron energy
    against n0 (1 + sin(pi x)) exp(-5 t) and exp(-10 t)
    (test/verification/MMS3/l2err/l2err.cpp:100-134,
    get_L2norm_error.py)."""
    info = vb.case_info("mms3")
    x = (np.arange(n) + 0.5) / n
    prof = 1e6 * (1.0 + np.sin(np.pi * x))
    ne, een = S[0], S[info["een_id"]]
    e1 = np.sqrt(np.mean((ne - prof * np.exp(-5.0 * t)) ** 2)) / np.mean(ne)
    e2 = np.sqrt(np.mean((een - prof * np.exp(-10.0 * t)) ** 2)) / np.mean(een)
    return float(e1), float(e2)
