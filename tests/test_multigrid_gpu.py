"""Multigrid solves on 3-D grids of several shapes and boundary combinations
against the oracle: several x/y/z thread blocks, non-cubic grids, a grid
whose coarsening stops at an odd size, Dirichlet/Neumann/periodic sides, two
and three smoothing iterations, and the FP32-refined form.

The FP64 solves converge to 1e-13 of the right-hand-side norm on both sides,
so the potentials agree to 1e-11 (the comparator's relative RMS,
py_utils/compare_fields_from_twoplotfiles.py:40-46) with V-cycle counts
within one of each other."""
import ctypes

import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

pytestmark = pytest.mark.gpu

TIGHT = dict(linsolve_reltol=1e-13, linsolve_abstol=0.0)


def rel(a, b):
    return field_error(b, a)[1]


def box(nx, ny, nz, pot_lo=(2, 2, 1), pot_hi=(2, 2, 1), **kw):
    cfg = W.townsend_config(3, nx)
    dx = 0.02 / nx
    cfg["n_cell"] = [nx, ny, nz]
    cfg["prob_hi"] = [0.02, dx * ny, dx * nz]
    cfg["pot_bc_lo"] = list(pot_lo)
    cfg["pot_bc_hi"] = list(pot_hi)
    for k, v in {**TIGHT, **kw}.items():
        cfg[k] = v
    return cfg


def pair(cfg, seed):
    state = W.initial_state(cfg, seed)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, state)
    o.set_state(0, state)
    return g, o


# (52, 52, 52) coarsens to 13^3, a level in natural (not red-black) layout
SHAPES = [(64, 64, 48), (96, 64, 32), (64, 96, 70), (52, 52, 52)]
BCS = [((2, 2, 1), (2, 2, 1)), ((1, 2, 2), (1, 2, 1)), ((1, 1, 1), (1, 1, 1))]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("bc", BCS)
def test_poisson_shapes_and_sides(require_gpu, shape, bc):
    g, o = pair(box(*shape, pot_lo=bc[0], pot_hi=bc[1]), 11)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    assert abs(sg.iterations - so.iterations) <= 1, (sg.iterations, so.iterations)
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-11


def test_poisson_periodic_sides(require_gpu):
    cfg = box(64, 32, 32, is_periodic=[1, 1, 0])
    cfg["pot_bc_lo"] = [0, 0, 1]
    cfg["pot_bc_hi"] = [0, 0, 1]
    g, o = pair(cfg, 12)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-11


@pytest.mark.parametrize("nu", [2, 3])
def test_smoothing_counts(require_gpu, nu):
    # (V(1,1) with piecewise-constant prolongation diverges on these grids,
    # on the GPU and in the oracle alike, so it is not a supported setting)
    cfg = box(64, 64, 64, linsolve_num_pre_smooth=nu, linsolve_num_post_smooth=nu)
    g, o = pair(cfg, 16)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    assert abs(sg.iterations - so.iterations) <= 1
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-11


@pytest.mark.parametrize("spec", [0, 1])
def test_species_solve_shapes(require_gpu, spec):
    cfg = box(64, 64, 48)
    g, o = pair(cfg, 13)
    o.solve_potential(0.0)
    g.set_state(0, o.get_state())
    ex = o.explicit_rhs(0.0)
    sg = g.implicit_solve_scalar(spec, ex, 0.0)
    so = o.implicit_solve_scalar(spec, ex, 0.0)
    assert sg.converged and so.converged
    assert rel(g.get_state(spec, 1), o.get_state(spec, 1)) < 1e-12


def test_fp32_refined_poisson_error(require_gpu):
    """FP32 V-cycles inside FP64 refinement to a 1e-10 relative residual:
    the potential within 1e-10 of the FP64-converged oracle (the precision
    target of the refined form)."""
    cfg = box(64, 64, 64, mg_precision=vb.VD_MG_FP32_REFINED)
    cfg["linsolve_reltol"] = 1e-10
    g = vb.Vidyut(cfg)
    ocfg = box(64, 64, 64)
    o = Oracle(ocfg)
    state = W.initial_state(cfg, 15)
    g.set_state(0, state)
    o.set_state(0, state)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-10


# Grids the oracle solves in seconds, with the level-size threshold of the
# sweeps built for HBM-resident levels lowered to one cell: every red-black
# level with nx % 4 == 0 then runs the two-planes-per-thread sweeps that
# otherwise only levels of 8 M cells or more use, FP64 and FP32, constant and
# face coefficients, with and without the fused prolongation.
BIG_SHAPES = [(64, 64, 48), (96, 64, 32), (64, 96, 70), (64, 64, 64)]


@pytest.mark.parametrize("shape", BIG_SHAPES)
@pytest.mark.parametrize("bc", BCS[:2])
def test_poisson_hbm_level_sweeps(require_gpu, monkeypatch, shape, bc):
    monkeypatch.setenv("VD_MG_BIG_LEVEL_CELLS", "1")
    g, o = pair(box(*shape, pot_lo=bc[0], pot_hi=bc[1]), 21)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    assert abs(sg.iterations - so.iterations) <= 1, (sg.iterations, so.iterations)
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-11


@pytest.mark.parametrize("spec", [0, 1])
def test_species_solve_hbm_level_sweeps(require_gpu, monkeypatch, spec):
    monkeypatch.setenv("VD_MG_BIG_LEVEL_CELLS", "1")
    cfg = box(64, 64, 64)
    g, o = pair(cfg, 22)
    o.solve_potential(0.0)
    g.set_state(0, o.get_state())
    ex = o.explicit_rhs(0.0)
    sg = g.implicit_solve_scalar(spec, ex, 0.0)
    so = o.implicit_solve_scalar(spec, ex, 0.0)
    assert sg.converged and so.converged
    assert rel(g.get_state(spec, 1), o.get_state(spec, 1)) < 1e-12


def test_fp32_refined_hbm_level_sweeps(require_gpu, monkeypatch):
    monkeypatch.setenv("VD_MG_BIG_LEVEL_CELLS", "1")
    cfg = box(64, 64, 64, mg_precision=vb.VD_MG_FP32_REFINED)
    cfg["linsolve_reltol"] = 1e-10
    g = vb.Vidyut(cfg)
    o = Oracle(box(64, 64, 64))
    state = W.initial_state(cfg, 23)
    g.set_state(0, state)
    o.set_state(0, state)
    sg = g.solve_potential(0.0)
    so = o.solve_potential(0.0)
    assert sg.converged and so.converged
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-10


@pytest.mark.parametrize("maxiter", [1, 3])
def test_poisson_stops_at_maxiter(require_gpu, maxiter):
    """A solve cut off by linsolve_maxiter: the convergence norm of each cycle
    is taken by the next cycle's first sweep, and the last cycle's by a
    standalone pass, so the result is exactly `maxiter` V-cycles, as in the
    oracle, and is reported as not converged."""
    cfg = box(64, 64, 64, linsolve_maxiter=maxiter)
    g, o = pair(cfg, 24)
    sg = vb.vd_solve_stats()
    assert vb.STATUS[g.lib.vd_poisson_solve(g.ctx, 0.0, ctypes.byref(sg))] == "VD_ERR_NOT_CONVERGED"
    so = o.solve_potential(0.0)
    assert not sg.converged and not so.converged
    assert sg.iterations == so.iterations == maxiter
    assert abs(sg.final_residual - so.final_residual) <= 1e-9 * so.final_residual
    pid = g.info["pot_id"]
    assert rel(g.get_state(pid, 1), o.get_state(pid, 1)) < 1e-12


# The TMA-staged sweeps (vd_mg_tma.cuh) against the register-staged ones on
# the same levels (threshold lowered to one cell, as above): the same cell
# arithmetic on the same neighbour values, so the same V-cycle count and the
# same bits.  Shapes with partial tiles in x (nx/2 < 64, not a multiple of
# 64) and y (ny not a multiple of 16), two tiles across x, odd plane counts
# per CTA; FP64 and the FP32-refined form (FP32 levels whose half-row is not
# a multiple of 16 bytes keep the register-staged sweep).
@pytest.mark.parametrize("shape", [(64, 64, 48), (72, 40, 36), (256, 32, 16), (96, 64, 70)])
@pytest.mark.parametrize("precision", [vb.VD_MG_FP64, vb.VD_MG_FP32_REFINED])
def test_tma_sweeps_equal_register_sweeps(require_gpu, monkeypatch, shape, precision):
    monkeypatch.setenv("VD_MG_BIG_LEVEL_CELLS", "1")
    runs = []
    for tma in ("1", "0"):
        monkeypatch.setenv("VD_MG_TMA", tma)
        cfg = box(*shape, mg_precision=precision)
        if precision == vb.VD_MG_FP32_REFINED:
            cfg["linsolve_reltol"] = 1e-10
        g = vb.Vidyut(cfg)
        g.set_state(0, W.initial_state(cfg, 31))
        st = g.solve_potential(0.0)
        runs.append((st.iterations, st.final_residual, g.get_state(g.info["pot_id"], 1)))
        g.close()
    assert runs[0][0] == runs[1][0] and runs[0][1] == runs[1][1]
    assert np.array_equal(runs[0][2], runs[1][2])


# Species face coefficients in one pass per species (k_species_faces3: each
# cell's diffusivity evaluated once) against one launch per direction
# (VD_SPECIES_FACES3=0): the same values and harmonic means, so the same
# solve bit for bit; periodic and walled sides, 3-D and 2-D, and the LMEA
# mechanism, whose diffusivities read the state.
@pytest.mark.parametrize("kind", ["box", "periodic", "2d", "lmea"])
def test_species_faces_one_pass_equal_per_direction(require_gpu, monkeypatch, kind):
    def make():
        if kind == "lmea":
            cfg = W.lmea_config(24)
            return cfg, W.lmea_state(cfg, 3)
        if kind == "2d":
            cfg = W.townsend_config(2, 64)
            return cfg, W.initial_state(cfg, 3)
        cfg = box(64, 40, 36) if kind == "box" else box(
            64, 40, 36, pot_lo=(0, 0, 1), pot_hi=(0, 0, 1))
        if kind == "periodic":
            cfg["is_periodic"] = [1, 1, 0]
            for key in ("eden", "ion", "neutral", "eenrg"):
                cfg[f"{key}_bc_lo"] = [0, 0, 2]
                cfg[f"{key}_bc_hi"] = [0, 0, 2]
        return cfg, W.initial_state(cfg, 3)

    runs = []
    for v in ("1", "0"):
        monkeypatch.setenv("VD_SPECIES_FACES3", v)
        cfg, S = make()
        g = vb.Vidyut(cfg)
        g.set_state(0, S)
        g.solve_potential(0.0, allow_unconverged=True)
        ex = g.explicit_rhs(0.0)
        out = []
        for spec in range(2):
            g.set_state(0, S)
            st = g.implicit_solve_scalar(spec, ex, 0.0, allow_unconverged=True)
            out.append((st.iterations, g.get_state(spec, 1)))
        g.step(2, allow_unconverged=True)
        out.append((0, g.get_state()))
        g.close()
        runs.append(out)
    for a, b in zip(*runs):
        assert a[0] == b[0] and np.array_equal(a[1], b[1])
