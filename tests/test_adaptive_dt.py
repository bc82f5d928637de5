"""Adaptive time step: Vidyut::find_time_scales and Vidyut::ComputeDt
(Source/TimeStep.cpp:14-134), switched on by vidyut.adaptive_dt.

CPU: the oracle's electron time scales against the published formulas
evaluated here with numpy on the same state (dt_edrift = min dx / max|mu_e||E|,
dt_ediff = 0.5 min dx^2 / max D_e / dim, dt_diel_relax = eps0 / e / max|mu_e| n_e),
and the step rule (CFL factors, dt_min/dt_max clamps, dt_stretch,
adaptive_dt_delay).  GPU: the library's step sizes, time scales and fields
against the oracle's over several adaptive steps."""
import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

EPS0 = 8.854187817e-12
ECHARGE = 1.60217662e-19
MU_E, D_E = 0.0382, 0.18  # townsend case electron mobility and diffusivity
TIGHT = dict(linsolve_reltol=1e-13, linsolve_abstol=0.0)


def case(dim=2, n=32, **kw):
    cfg = W.townsend_config(dim, n)
    cfg["adaptive_dt"] = 1
    for k, v in {**TIGHT, **kw}.items():
        cfg[k] = v
    return cfg


def state_with_field(cfg, seed=5):
    """The seeded blobs plus a seeded cell field, so that the drift scale is
    defined from the first step."""
    S = W.initial_state(cfg, seed)
    info = vb.case_info(cfg.case)
    rng = np.random.default_rng(seed)
    for d in range(cfg["dim"]):
        S[info["efx_id"] + d] = rng.normal(0.0, 2e6, S[0].shape)
    return S


def expected_scales(cfg, S):
    info = vb.case_info(cfg.case)
    dim = cfg["dim"]
    dx = [(cfg["prob_hi"][d] - cfg["prob_lo"][d]) / cfg["n_cell"][d] for d in range(dim)]
    esum = np.zeros_like(S[0])
    for d in range(dim):
        e = S[info["efx_id"] + d]
        esum = esum + e * e
    emag = np.sqrt(esum)
    vmax = float(np.max(MU_E * emag))
    nmax = float(np.max(MU_E * S[0]))
    big = np.finfo(np.float64).max
    t_drift = min(dx[d] / vmax for d in range(dim)) if vmax > 0 else big
    t_diff = min(0.5 * dx[d] * dx[d] / D_E / dim for d in range(dim))
    t_diel = EPS0 / ECHARGE / nmax
    return t_drift, t_diff, t_diel


def close(a, b, tol=1e-14):
    return abs(a - b) <= tol * abs(b)


def test_oracle_time_scales_match_formulas():
    cfg = case()
    S = state_with_field(cfg)
    o = Oracle(cfg)
    o.set_state(0, S)
    st = o.step(1)
    t_drift, t_diff, t_diel = expected_scales(cfg, S)
    assert close(st.dt_edrift, t_drift), (st.dt_edrift, t_drift)
    assert close(st.dt_ediff, t_diff), (st.dt_ediff, t_diff)
    assert close(st.dt_diel_relax, t_diel), (st.dt_diel_relax, t_diel)
    # the first step starts at time 0, not past adaptive_dt_delay = 0: the
    # fixed step (Source/TimeStep.cpp:22)
    assert st.dt == cfg["dt"]
    S1 = o.get_state()
    st = o.step(1)
    t_drift, t_diff, t_diel = expected_scales(cfg, S1)
    assert close(st.dt_edrift, t_drift) and close(st.dt_diel_relax, t_diel)
    want = min(0.7 * t_drift, 1.0 * t_diff, 1.0 * t_diel)
    want = min(max(want, 1e-14), 1e-9)
    assert close(st.dt, want)
    assert close(st.time, cfg["dt"] + want)


def test_oracle_step_rules():
    # (each first step is the fixed one: time 0 is not past the delay)
    # dt_max clamps from above
    cfg = case(dt_max=1e-13)
    S = state_with_field(cfg)
    o = Oracle(cfg)
    o.set_state(0, S)
    assert o.step(1).dt == cfg["dt"]
    assert o.step(1).dt == 1e-13
    # dt_min clamps from below
    cfg = case(dt_min=1e-6, dt_max=1e-5)
    o = Oracle(cfg)
    o.set_state(0, S)
    o.step(1)
    assert o.step(1).dt == 1e-6
    # dt_stretch limits the growth from the previous step
    cfg = case(dt=1e-14, dt_stretch=1.5)
    o = Oracle(cfg)
    o.set_state(0, S)
    assert o.step(1).dt == 1e-14
    st2 = o.step(1)
    assert close(st2.dt, 1.5e-14)
    st3 = o.step(1)
    assert close(st3.dt, 1.5 * 1.5e-14)
    assert close(st3.time, 1e-14 + 1.5e-14 + 2.25e-14)
    # adaptive_dt_delay: the fixed step until the time passes the delay
    cfg = case(dt=1e-13, adaptive_dt_delay=1.5e-13)
    o = Oracle(cfg)
    o.set_state(0, S)
    assert o.step(1).dt == 1e-13
    assert o.step(1).dt == 1e-13  # time 1e-13, not past the delay
    st = o.step(1)                # time 2e-13 > delay
    assert st.dt != 1e-13
    # without transport only the dielectric scale limits the step
    cfg = case(do_transport=0)
    o = Oracle(cfg)
    o.set_state(0, S)
    o.step(1)
    st = o.step(1)
    assert close(st.dt, min(max(st.dt_diel_relax, 1e-14), 1e-9))


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,steps", [(2, 64, 4), (3, 32, 3)])
def test_adaptive_dt_parity(require_gpu, dim, n, steps):
    cfg = case(dim, n, advective_cfl=0.5, dt_stretch=1.2)
    S = W.initial_state(cfg, 6)  # zero field: the first step has no drift scale
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S)
    o.set_state(0, S)
    info = g.info
    for s in range(steps):
        sg = g.step(1)
        so = o.step(1)
        # step 0 reads the common initial state; later steps read states that
        # agree to the field tolerance below, and the scales are max-norms of
        # them
        tol = 1e-14 if s == 0 else 1e-11
        for a, b in ((sg.dt, so.dt), (sg.dt_ediff, so.dt_ediff),
                     (sg.dt_diel_relax, so.dt_diel_relax), (sg.dt_edrift, so.dt_edrift),
                     (sg.time, so.time)):
            assert abs(a - b) <= tol * abs(b), (s, a, b)
        Sg, So = g.get_state(), o.get_state()
        for c in (0, 1, info["pot_id"]):
            r = field_error(So[c], Sg[c])[1]
            assert r < 1e-11, (s, c, r)
