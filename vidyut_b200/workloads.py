"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every input is generated on the host from a
fixed seed and copied bit-identically to the CUDA library and to the CPU
oracle.  Configurations (two-species Townsend discharge, background gas
N = 2.45e25 m^-3 at 300 K, WENO5-Z drift flux):

* ``townsend_2d``: 2-D, 1 cm x 1 cm, 0 V bottom / 20 kV top (Dirichlet on y),
  Neumann sides, one seeded Gaussian (peak 1e18 m^-3, sigma 0.5 mm) on a
  1e13 m^-3 background, dt = 1e-12 s.
* ``townsend_3d``: 3-D, 2 cm cube, 20 kV across z, Neumann on x and y, five
  seeded Gaussian blobs (peak log-uniform 1e16-1e19 m^-3, sigma uniform
  0.3-1 mm, centres uniform in the middle 60 % of the box), dt = 5e-13 s.
"""
from __future__ import annotations

import numpy as np

from . import Config, case_info

NGAS = 2.45e25
TGAS = 300.0
K_B = 1.380649e-23
TE_LFA = 5802.25


def _common(cfg: Config):
    cfg["hyp_order"] = 5
    cfg["weno_scheme"] = 3
    cfg["using_LFA"] = 1
    cfg["bound_specden"] = 1
    cfg["gas_temperature"] = TGAS
    cfg["gas_pressure"] = NGAS * K_B * TGAS
    cfg.set("vidyut.bg_species_ids", "2")


def townsend_config(dim: int, n: int, **kw) -> Config:
    cfg = Config("townsend")
    cfg["dim"] = dim
    _common(cfg)
    if dim == 2:
        cfg["n_cell"] = [n, n, 1]
        cfg["prob_hi"] = [0.01, 0.01, 1.0]
        cfg["dt"] = 1e-12
        bc_pot_lo, bc_pot_hi = [2, 1, 2], [2, 1, 2]
        cfg["voltage_amp_hi"] = [0.0, 20e3, 0.0]
    else:
        cfg["n_cell"] = [n, n, n]
        cfg["prob_hi"] = [0.02, 0.02, 0.02]
        cfg["dt"] = 5e-13
        bc_pot_lo, bc_pot_hi = [2, 2, 1], [2, 2, 1]
        cfg["voltage_amp_hi"] = [0.0, 0.0, 20e3]
    cfg["pot_bc_lo"] = bc_pot_lo
    cfg["pot_bc_hi"] = bc_pot_hi
    for k, v in kw.items():
        cfg[k] = v
    return cfg


def blobs(dim: int, seed: int, L: float):
    """Blob centres, peaks and widths of the seeded initial state."""
    rng = np.random.default_rng(seed)
    if dim == 2:
        c = rng.uniform(0.3 * L, 0.7 * L, size=(1, 2))
        return c, np.array([1e18]), np.array([0.5e-3])
    c = rng.uniform(0.2 * L, 0.8 * L, size=(5, 3))
    peak = 10.0 ** rng.uniform(16.0, 19.0, size=5)
    sig = rng.uniform(0.3e-3, 1.0e-3, size=5)
    return c, peak, sig


def initial_state(cfg: Config, seed: int = 0) -> np.ndarray:
    """Full NVAR-component initial state, shape (nvar, nz, ny, nx)."""
    info = case_info(cfg.case)
    dim = cfg["dim"]
    nx, ny = cfg["n_cell"][0], cfg["n_cell"][1]
    nz = cfg["n_cell"][2] if dim == 3 else 1
    L = cfg["prob_hi"][0] - cfg["prob_lo"][0]
    dx = L / nx
    x = cfg["prob_lo"][0] + (np.arange(nx) + 0.5) * dx
    y = cfg["prob_lo"][1] + (np.arange(ny) + 0.5) * dx
    centres, peak, sig = blobs(dim, seed, L)
    n = np.full((nz, ny, nx), 1e13)
    if dim == 2:
        X, Y = np.meshgrid(x, y, indexing="xy")
        for (cx, cy), a, s in zip(centres, peak, sig):
            n[0] += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    else:
        z = cfg["prob_lo"][2] + (np.arange(nz) + 0.5) * dx
        for (cx, cy, cz), a, s in zip(centres, peak, sig):
            gx = np.exp(-((x - cx) ** 2) / (2 * s * s))
            gy = np.exp(-((y - cy) ** 2) / (2 * s * s))
            gz = np.exp(-((z - cz) ** 2) / (2 * s * s))
            n += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    S = np.zeros((info["nvar"], nz, ny, nx))
    S[0] = n
    S[1] = n
    S[2] = NGAS
    S[info["etemp_id"]] = TE_LFA
    S[info["een_id"]] = 1.5 * n * K_B * TE_LFA
    S[info["cmask_id"]] = 1.0
    return S
