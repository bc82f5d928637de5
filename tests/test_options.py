"""Reference options on the step's path that the benchmark workloads leave
at their defaults:

* the default thermal-flux species wall (boundary code 3, inhomogeneous
  Neumann, plasmachem_transport::species_bc, Source/PlasmaChem.H:75-200)
  for every branch of that callback: electrons, electron energy, positive
  and negative ions (drift out of the wall or none), transported neutrals;
* the applied-voltage profiles 1 (sinusoid) and 2 (single triangle) of
  get_applied_potential (Source/HelperFuncs.H:125-161);
* background-species chemistry (vidyut.do_bg_reactions,
  Source/Evolve.cpp:432-456): the background density advanced by dt times
  its reaction source and floored.

The oracle carries its own restatement of the default callbacks
(oracle/oracle_defaults.H), so the GPU tests compare two independent
readings of Source/PlasmaChem.H.  The CPU tests check the oracle against a
numpy restatement of the reference formula."""
import math

import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

TIGHT = dict(linsolve_reltol=1e-13, linsolve_abstol=0.0)


def rel(a, b):
    return field_error(b, a)[1]


def applied_potential(t, end, vprof, v1, v2, vfreq, vdur, vcen):
    """get_applied_potential (Source/HelperFuncs.H:125-161)."""
    amp = v1 if end == -1 else v2
    if vprof == 1:
        return math.sin(2.0 * math.pi * vfreq * t) * amp
    if vprof == 2:
        if t <= vcen:
            return (1.0 - (vcen - t) / (vdur / 2.0)) * amp if vcen - t < vdur / 2.0 else 0.0
        return (1.0 - (t - vcen) / (vdur / 2.0)) * amp if t - vcen < vdur / 2.0 else 0.0
    return amp


def voltage_cfg(profile, n=32):
    cfg = W.townsend_config(2, n, do_spacechrg=0, voltage_profile=profile, **TIGHT)
    cfg["voltage_amp_lo"] = [0.0, 3e3, 0.0]
    cfg["voltage_amp_hi"] = [0.0, 20e3, 0.0]
    cfg["voltage_freq"] = 13.56e6
    cfg["voltage_center"] = 4e-9
    cfg["voltage_dur"] = 6e-9
    return cfg


# times on the sinusoid and on both flanks of the triangle, its peak and
# outside the pulse
TIMES = [0.0, 1.3e-9, 2.0e-9, 3.1e-9, 4e-9, 5.2e-9, 6.9e-9, 8e-9]


@pytest.mark.parametrize("profile", [0, 1, 2])
def test_oracle_voltage_profiles_linear_potential(profile):
    """Without space charge the potential between the Dirichlet plates is
    linear, which the second-order discretisation reproduces exactly:
    phi(y_j) = V_lo + (V_hi - V_lo) y_j / L with the face values from
    get_applied_potential at the solve's time."""
    cfg = voltage_cfg(profile)
    c = cfg.c
    n = cfg["n_cell"][1]
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 1))
    y = (np.arange(n) + 0.5) / n
    pid = o.info["pot_id"]
    for t in TIMES:
        o.solve_potential(t)
        vlo = applied_potential(t, -1, profile, c.voltage_amp_lo[1], c.voltage_amp_hi[1],
                                c.voltage_freq, c.voltage_dur, c.voltage_center)
        vhi = applied_potential(t, +1, profile, c.voltage_amp_lo[1], c.voltage_amp_hi[1],
                                c.voltage_freq, c.voltage_dur, c.voltage_center)
        phi = o.get_state(pid, 1)[0, 0]          # (ny, nx)
        want = vlo + (vhi - vlo) * y
        scale = max(abs(vlo), abs(vhi), 1.0)
        assert np.max(np.abs(phi.mean(axis=1) - want)) <= 1e-9 * scale, (t, vlo, vhi)


@pytest.mark.gpu
@pytest.mark.parametrize("profile", [1, 2])
def test_voltage_profiles_parity(require_gpu, profile):
    cfg = voltage_cfg(profile)
    cfg["do_spacechrg"] = 1
    S0 = W.initial_state(cfg, 2)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    pid = g.info["pot_id"]
    for t in TIMES:
        g.set_state(0, S0)
        o.set_state(0, S0)
        g.solve_potential(t)
        o.solve_potential(t)
        a, b = g.get_state(pid, 1), o.get_state(pid, 1)
        if np.max(np.abs(b)) == 0.0:
            assert np.max(np.abs(a)) == 0.0
        else:
            assert rel(a, b) < 1e-11, (t, rel(a, b))
    # a step at a time inside the triangle: the step's solves see t
    g.set_state(0, S0)
    o.set_state(0, S0)
    g.set_time(3.1e-9, 0)
    o.set_time(3.1e-9, 0)
    g.step(2)
    o.step(2)
    Sg, So = g.get_state(), o.get_state()
    for comp in (0, 1, pid):
        assert rel(Sg[comp], So[comp]) < 1e-11, (comp, rel(Sg[comp], So[comp]))


def wall_cfg(n=20, **kw):
    """The LMEA mechanism (electrons, four positive ions, a negative ion, a
    background neutral and a transported neutral, with the electron energy
    equation) between thermal-flux walls on z (code 3), so that every branch
    of the default species callback runs; the potential keeps its plates."""
    cfg = W.lmea_config(n, **TIGHT)
    for key in ("eden", "eenrg", "ion", "neutral"):
        cfg[f"{key}_bc_lo"] = [2, 2, 3]
        cfg[f"{key}_bc_hi"] = [2, 2, 3]
    for k, v in kw.items():
        cfg[k] = v
    return cfg


@pytest.mark.gpu
def test_thermal_flux_walls_parity(require_gpu):
    cfg = wall_cfg()
    S0 = W.lmea_state(cfg, 11)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S0)
    o.set_state(0, S0)
    info = g.info
    for s in range(2):
        g.step(1)
        o.step(1)
        Sg, So = g.get_state(), o.get_state()
        for comp in [0, 1, 2, 3, 4, 5, 7, info["een_id"], info["etemp_id"], info["pot_id"]]:
            r = rel(Sg[comp], So[comp])
            assert r < 1e-11, (s, comp, r)
    # the walls drain particles: the wall cells differ from a run with
    # homogeneous Neumann walls, so the flux path was taken
    h = wall_cfg()
    for key in ("eden", "eenrg", "ion", "neutral"):
        h[f"{key}_bc_lo"] = [2, 2, 2]
        h[f"{key}_bc_hi"] = [2, 2, 2]
    gh = vb.Vidyut(h)
    gh.set_state(0, S0)
    gh.step(2)
    Sh = gh.get_state()
    assert rel(Sg[0][0], Sh[0][0]) > 1e-9 and rel(Sg[7][-1], Sh[7][-1]) > 1e-12


@pytest.mark.gpu
def test_implicit_diffusion_thermal_flux_wall_parity(require_gpu):
    """One species solve per branch of the wall callback, on the same
    explicit sources, through vd_implicit_diffusion."""
    cfg = wall_cfg()
    S0 = W.lmea_state(cfg, 12)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    o.set_state(0, S0)
    o.solve_potential(0.0)
    S = o.get_state()
    ex = o.explicit_rhs(0.0)
    een = g.info["een_id"]
    for spec in (0, een, 1, 5, 7):
        g.set_state(0, S)
        o.set_state(0, S)
        sg = g.implicit_solve_scalar(spec, ex, 0.0)
        so = o.implicit_solve_scalar(spec, ex, 0.0)
        assert sg.converged and so.converged
        assert rel(g.get_state(spec, 1), o.get_state(spec, 1)) < 1e-12, spec


@pytest.mark.gpu
def test_background_reactions_parity(require_gpu):
    cfg = W.lmea_config(20, do_bg_reactions=1, **TIGHT)
    S0 = W.lmea_state(cfg, 13)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S0)
    o.set_state(0, S0)
    for s in range(2):
        g.step(1)
        o.step(1)
    Sg, So = g.get_state(), o.get_state()
    # the background neutral (component 6) moved by its reaction source
    assert rel(Sg[6], S0[6]) > 1e-14
    for comp in (0, 1, 6, 7, g.info["pot_id"]):
        r = rel(Sg[comp], So[comp])
        assert r < 1e-11, (comp, r)
    # without the switch the background stays put
    cfg0 = W.lmea_config(20, **TIGHT)
    g0 = vb.Vidyut(cfg0)
    g0.set_state(0, S0)
    g0.step(2)
    assert np.array_equal(g0.get_state(6, 1)[0], S0[6])
