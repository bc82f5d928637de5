"""GPU test of vd_poisson_solve_noalloc, the Poisson solve that allocates no
device memory (for callers that must not allocate while they run, e.g. a
host framework whose own pool owns the device).  It is called through the
C ABI on caller-owned device arrays and must reproduce the context-based
field solve (vd_poisson_solve) to the parity tolerance of the other Poisson
tests, on two calls in a row that share its built-in scratch.  The file is
named to be collected last."""
import ctypes as C

import numpy as np
import pytest

import vidyut_b200 as vb
from vidyut_b200 import workloads as W

pytestmark = pytest.mark.gpu

ECHARGE = 1.60217662e-19
EPS0 = 8.854187817e-12


def _i3(v):
    return (C.c_int * 3)(*v)


def _d3(v):
    return (C.c_double * 3)(*v)


def noalloc_solve(lib, cfg, rhs_dev, phi_dev):
    n = cfg["n_cell"]
    dx = [(cfg["prob_hi"][d] - cfg["prob_lo"][d]) / n[d] for d in range(3)]
    st = vb.vd_solve_stats()
    err = C.create_string_buffer(256)
    rc = lib.vd_poisson_solve_noalloc(
        3, _i3(n), _d3(dx), _i3(cfg["pot_bc_lo"]), _i3(cfg["pot_bc_hi"]),
        _d3(cfg["voltage_amp_lo"]), _d3(cfg["voltage_amp_hi"]),
        C.c_void_p(rhs_dev.data_ptr()), C.c_void_p(phi_dev.data_ptr()),
        cfg["linsolve_reltol"], cfg["linsolve_abstol"], cfg["linsolve_maxiter"],
        C.byref(st), err, 256)
    return rc, st, err.value.decode()


def field_rhs(state):
    # the context path's right-hand side: -(e/eps0) sum_s q_s n_s with the
    # charges E -1, ION +1 (potential_scale 1)
    r = 0.0 + (-1.0) * state[0]
    r = r + 1.0 * state[1]
    return r * (-ECHARGE / EPS0)


def test_noalloc_poisson_matches_context_solve(require_gpu):
    import torch

    cfg = W.townsend_config(3, 32)
    cfg["linsolve_reltol"] = 1e-13
    cfg["linsolve_abstol"] = 0.0
    g = vb.Vidyut(cfg)
    pot = g.info["pot_id"]
    phi_dev = torch.zeros((32, 32, 32), dtype=torch.float64, device="cuda")
    for seed in (11, 12):  # two calls in a row through the same scratch
        state = W.initial_state(cfg, seed)
        g.set_state(0, state)
        g.solve_potential(0.0)
        ref = g.get_state(pot, 1)[0]
        rhs_dev = torch.tensor(field_rhs(state), dtype=torch.float64, device="cuda")
        phi_dev.zero_()
        rc, st, msg = noalloc_solve(g.lib, cfg, rhs_dev, phi_dev)
        assert rc == 0, msg
        assert st.converged and st.iterations > 0
        got = phi_dev.cpu().numpy()
        rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert rel < 1e-11, (seed, rel)
    g.close()


def test_noalloc_poisson_rejects_grids_beyond_its_scratch(require_gpu):
    import torch

    cfg = W.townsend_config(3, 256)
    rhs_dev = torch.zeros((256, 256, 256), dtype=torch.float64, device="cuda")
    phi_dev = torch.zeros_like(rhs_dev)
    rc, _, msg = noalloc_solve(vb.load("townsend"), cfg, rhs_dev, phi_dev)
    assert rc == 1
    assert "at most" in msg
    assert float(phi_dev.abs().max()) == 0.0
