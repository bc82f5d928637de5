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
