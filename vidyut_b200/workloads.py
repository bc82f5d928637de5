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
* ``lmea``: the 8-species LMEA mechanism of ``vidyut_b200/mechgen.py``
  (seed 2) with the electron-energy equation, 2 cm cube, 20 kV across z,
  dt = 1e-12 s; initial ion, negative-ion and excited-neutral densities are
  log-uniform 1e10-1e18 m^-3 per species, modulated by a smooth seeded
  field, electrons set for quasi-neutrality, Te = 1 eV.
* ``adjoint``: the ``lmea`` state with frozen analytic fields for the discrete
  adjoint: E along -z of 1e6 V/m (times a smooth seeded factor in 0.5-1.5,
  plus x/y components of a tenth of that), Te = 1 eV times a smooth seeded
  factor in 0.75-1.25; gradients by the explicit flux + source steps at
  dt = 1e-12 s.
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


TE_1EV = 11604.518


def lmea_config(n: int, **kw) -> Config:
    cfg = Config("lmea8")
    cfg["dim"] = 3
    cfg["n_cell"] = [n, n, n]
    cfg["prob_hi"] = [0.02, 0.02, 0.02]
    cfg["dt"] = 1e-12
    cfg["hyp_order"] = 5
    cfg["weno_scheme"] = 3
    cfg["elecenergy_solve"] = 1
    cfg["bound_specden"] = 1
    cfg["min_species_density"] = 1.0
    cfg["gas_temperature"] = TGAS
    cfg["gas_pressure"] = NGAS * K_B * TGAS
    cfg.set("vidyut.bg_species_ids", "6")
    cfg["pot_bc_lo"] = [2, 2, 1]
    cfg["pot_bc_hi"] = [2, 2, 1]
    cfg["voltage_amp_hi"] = [0.0, 0.0, 20e3]
    for k, v in kw.items():
        cfg[k] = v
    return cfg


def lmea_state(cfg: Config, seed: int = 0) -> np.ndarray:
    info = case_info(cfg.case)
    nx, ny, nz = cfg["n_cell"]
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz

    def smooth():
        f = np.zeros((nz, ny, nx))
        for _ in range(3):
            kx, ky, kz = rng.integers(1, 4, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            f += (np.cos(2 * np.pi * kz * z + ph[2])[:, None, None]
                  * np.cos(2 * np.pi * ky * y + ph[1])[None, :, None]
                  * np.cos(2 * np.pi * kx * x + ph[0])[None, None, :])
        return 1.0 + 0.25 * f

    S = np.zeros((info["nvar"], nz, ny, nx))
    pos = [1, 2, 3, 4]
    for s in pos:
        S[s] = 10.0 ** rng.uniform(10.0, 18.0) * smooth()
    S[5] = 0.5 * S[pos].sum(axis=0) * 10.0 ** rng.uniform(-8.0, 0.0)
    S[0] = S[pos].sum(axis=0) - S[5]
    S[6] = NGAS
    S[7] = 10.0 ** rng.uniform(10.0, 18.0) * smooth()
    S[info["etemp_id"]] = TE_1EV
    S[info["een_id"]] = 1.5 * S[0] * K_B * TE_1EV
    S[info["cmask_id"]] = 1.0
    return S


def adjoint_config(n: int, **kw) -> Config:
    """The LMEA case as the adjoint runs it (clamped ghost cells, every
    species BC Neumann so no wall zeroes a flux)."""
    return lmea_config(n, **kw)


def adjoint_state(cfg: Config, seed: int = 0, efield: float = 1e6) -> np.ndarray:
    """``lmea_state`` plus the frozen E and Te fields of the adjoint runs."""
    info = case_info(cfg.case)
    S = lmea_state(cfg, seed)
    nx, ny, nz = cfg["n_cell"]
    rng = np.random.default_rng(seed + 1000)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz

    def wave():
        kx, ky, kz = rng.integers(1, 3, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        return (np.cos(2 * np.pi * kz * z + ph[2])[:, None, None]
                * np.cos(2 * np.pi * ky * y + ph[1])[None, :, None]
                * np.cos(2 * np.pi * kx * x + ph[0])[None, None, :])

    ez = -efield * (1.0 + 0.5 * wave())
    S[info["efx_id"]] = 0.1 * efield * wave()
    S[info["efx_id"] + 1] = 0.1 * efield * wave()
    S[info["efx_id"] + 2] = ez
    S[info["etemp_id"]] = TE_1EV * (1.0 + 0.25 * wave())
    return S


def mgsolve_config(n: int, **kw) -> Config:
    """Mixed-precision Poisson and implicit-diffusion workload: unit cube,
    n^3 cells, 7-point Laplacian, Dirichlet (0 V) on the z faces and
    homogeneous Neumann on x and y, for the potential and the diffusing
    ion alike; implicit diffusion at dt = 1e-11 s."""
    cfg = Config("mgsolve")
    cfg["dim"] = 3
    cfg["n_cell"] = [n, n, n]
    cfg["prob_hi"] = [1.0, 1.0, 1.0]
    cfg["dt"] = 1e-11
    cfg["do_reactions"] = 0
    cfg["bound_specden"] = 0
    for key in ("pot", "eden", "ion", "neutral", "eenrg"):
        cfg[f"{key}_bc_lo"] = [2, 2, 1]
        cfg[f"{key}_bc_hi"] = [2, 2, 1]
    for k, v in kw.items():
        cfg[k] = v
    return cfg


def mgsolve_fields(cfg: Config, seed: int = 0):
    """Electron density, ion density and ion diffusivity of the solver
    workload, each (nz, ny, nx): net charge n_ion - n_e of eight seeded
    Gaussians of amplitude +-1e16 m^-3 (random sign, centres uniform in the
    middle 80 % of the cube, sigma uniform in 0.03-0.1 of the edge) plus
    white noise of 1e-3 of that amplitude, on a uniform 1e17 m^-3 electron
    background; diffusivity log-uniform in 1e-6-1e-1 m^2/s cell by cell."""
    nx, ny, nz = cfg["n_cell"]
    rng = np.random.default_rng(seed)
    amp = 1e16
    c = rng.uniform(0.1, 0.9, size=(8, 3))
    sg = rng.uniform(0.03, 0.1, size=8)
    sgn = rng.choice([-1.0, 1.0], size=8)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    rho = np.zeros((nz, ny, nx))
    for b in range(8):
        gx = np.exp(-((x - c[b, 0]) ** 2) / (2 * sg[b] ** 2))
        gy = np.exp(-((y - c[b, 1]) ** 2) / (2 * sg[b] ** 2))
        gz = np.exp(-((z - c[b, 2]) ** 2) / (2 * sg[b] ** 2))
        rho += (sgn[b] * amp) * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    rho += 1e-3 * amp * rng.standard_normal(size=rho.shape)
    ne = np.full((nz, ny, nx), 1e17)
    nion = rho
    nion += 1e17
    D = 10.0 ** rng.uniform(-6.0, -1.0, size=rho.shape)
    return ne, nion, D


def mgsolve_state(cfg: Config, seed: int = 0) -> np.ndarray:
    """The full state of the solver workload (mgsolve_fields, with the ion
    diffusivity in the electron-temperature slot, see
    cases/mgsolve/Chemistry.H)."""
    info = case_info(cfg.case)
    ne, nion, D = mgsolve_fields(cfg, seed)
    S = np.zeros((info["nvar"],) + ne.shape)
    S[0] = ne
    S[1] = nion
    S[info["etemp_id"]] = D
    S[info["cmask_id"]] = 1.0
    return S


def mgsolve_load(g, cfg: Config, seed: int = 0) -> None:
    """Copy the solver workload into a context component by component (at
    512^3 the full state would be 27 GB of host memory; the context starts
    from an all-zero state)."""
    info = case_info(cfg.case)
    ne, nion, D = mgsolve_fields(cfg, seed)
    g.set_state(0, ne)
    g.set_state(1, nion)
    g.set_state(info["etemp_id"], D)
    D.fill(1.0)
    g.set_state(info["cmask_id"], D)
