"""Semi-implicit electron-Poisson coupling (vidyut.electron_poisson_coupling,
Source/Evolve.cpp:281-352, Source/PotentialSolve.cpp:262-347): the electron
solve precedes the potential solve, whose operator carries
b = -(1 + dt/tau_diel), tau_diel = |eps0 / (e mu_e n_e)|, and whose right-hand
side carries ((n_e^new - n_e^old)/dt - S_expl + S_rxn) dt e / eps0; the pair is
repeated electron_poisson_maxiters times.

CPU (oracle): for dt -> 0 the coupled step approaches the plain one (the
coupling terms are O(dt)); the electron/potential iteration contracts (the
change from 2 to 3 iterations is well below the change from 1 to 2).
GPU: the library against the oracle, 1 and 2 iterations, 2-D and 3-D."""
import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

TIGHT = dict(linsolve_reltol=1e-13, linsolve_abstol=0.0)


def case(dim, n, **kw):
    cfg = W.townsend_config(dim, n)
    for k, v in {**TIGHT, **kw}.items():
        cfg[k] = v
    return cfg


def run_oracle(cfg, S, steps=1):
    o = Oracle(cfg)
    o.set_state(0, S)
    o.step(steps)
    return o.get_state()


def rel(a, b):
    return field_error(b, a)[1]


def test_oracle_coupling_vanishes_with_dt():
    """The coupled and plain steps differ by O(dt): the difference falls by
    the same factor as dt (100x here), for the potential and the electrons."""
    pot = vb.case_info("townsend")["pot_id"]
    diffs = []
    for dt in (1e-15, 1e-17):
        cfg0 = case(2, 32, dt=dt)
        cfg1 = case(2, 32, dt=dt, electron_poisson_coupling=1)
        S = W.initial_state(cfg0, 9)
        a, b = run_oracle(cfg0, S), run_oracle(cfg1, S)
        diffs.append((rel(b[pot], a[pot]), rel(b[0], a[0])))
    for q in range(2):
        assert diffs[0][q] > 0
        assert abs(diffs[1][q] / diffs[0][q] - 1e-2) < 1e-3, diffs


def test_oracle_coupling_iteration_contracts():
    pot = vb.case_info("townsend")["pot_id"]
    S = W.initial_state(case(2, 32), 10)
    r = [run_oracle(case(2, 32, electron_poisson_coupling=1, electron_poisson_maxiters=m), S)
         for m in (1, 2, 3)]
    d12 = rel(r[1][pot], r[0][pot])
    d23 = rel(r[2][pot], r[1][pot])
    assert d12 > 0 and d23 < 0.1 * d12, (d12, d23)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,iters", [(2, 64, 1), (2, 64, 2), (3, 32, 1)])
def test_coupling_parity(require_gpu, dim, n, iters):
    cfg = case(dim, n, electron_poisson_coupling=1, electron_poisson_maxiters=iters)
    S = W.initial_state(cfg, 11)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S)
    o.set_state(0, S)
    info = g.info
    for s in range(3):
        g.step(1)
        o.step(1)
        Sg, So = g.get_state(), o.get_state()
        # The coupling source holds (n_e^new - n_e^old)/dt, a difference of
        # nearly equal densities: once n_e^new or n_e^old carries the
        # 1e-12-level solver rounding by which the two sides differ (from the
        # second step on, or from the second electron/potential iteration),
        # it is amplified by n_e / dn_e (~1e3 here) in the potential.  The
        # first single-iteration step starts from the common state and holds
        # every field to 1e-10.
        tight = s == 0 and iters == 1
        for c, tol in ((0, 1e-10), (1, 1e-10), (info["pot_id"], 1e-10 if tight else 1e-8),
                       (info["etemp_id"], 1e-10)):
            r = rel(Sg[c], So[c])
            assert r < tol, (s, c, r)
