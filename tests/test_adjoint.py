"""Discrete adjoint of N explicit flux + source steps (no reference
counterpart; the reference computes no sensitivities).

Objective: total electron count after the last step.  Parameters: the 30
log pre-factor shifts of the LMEA mechanism and the electron mobility scale.
Checks, all FP64:
* the oracle's tangent-linear pass against central differences of its own
  forward map (CPU);
* the library's forward map against the oracle's, species by species
  (relative L2 <= 1e-12, pointwise FP64 arithmetic on both sides);
* the library's adjoint gradient against the oracle's tangent-linear
  gradient (<= 1e-9 relative: both are exact derivatives of the same map and
  differ by rounding only);
* the library's adjoint gradient against central finite differences of the
  library's own forward map: |g - fd| <= 1e-6 |fd| + 4 eps |J| / h.  The
  second term is the differences' own rounding floor (J(p +- h) each carry
  a relative rounding error of order eps = 2.2e-16); where the objective
  moves by only ~1e-4 of itself per unit parameter, as in these short runs,
  that floor is comparable to 1e-6 of the gradient at h = 1e-6, so the small
  cases use h = 1e-3 (truncation error h^2/6 of the third derivative, ~2e-7
  relative for the exponential pre-factor dependence) and the 128^3 workload
  uses central differences at h = 1e-6 with the rounding of J as their
  floor and cell-by-cell differences at h = 1e-4 that resolve 1e-6
  relative (test_adjoint_c4_vs_fd);
* checkpoint intervals that do and do not divide the step count give the same
  gradient; the same checks through a torch.autograd.Function wrapper (test
  harness only);
* the line-march kernels against the one-thread-per-face and per-cell forms
  they replace (VD_ADJ_FACES_LINE=0, VD_ADJ_STEP_LINE=0) and across segment
  counts (VD_ADJ_LINE_SEGMENTS), on a box, a periodic direction with
  flux-zeroing walls, and 2-D, each also against the oracle's tangent-linear
  gradient.
"""
import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W

NR = 30


def small_case(n=12, seed=3, dt=5e-12):
    """A box of 0.2 mm so that the drift moves the electrons by a visible
    fraction of a cell within a few steps (CFL ~ 0.2 per step at 5 MV/m)."""
    cfg = W.adjoint_config(n, prob_hi=[2e-4, 2e-4, 2e-4], dt=dt)
    S = W.adjoint_state(cfg, seed, efield=5e6)
    return cfg, S


def params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NR + 1)
    p[:NR] = rng.uniform(-0.2, 0.2, NR)
    p[NR] = 1.1
    return p


def unit(k):
    e = np.zeros(NR + 1)
    e[k] = 1.0
    return e


EPS = np.finfo(np.float64).eps


def fd_ok(g, fd, J, h):
    return abs(g - fd) <= 1e-6 * abs(fd) + 4 * EPS * abs(J) / h


def grad_close(g, ref, rtol):
    floor = 1e-6 * np.max(np.abs(ref))
    err = np.abs(g - ref) / np.maximum(np.abs(ref), floor)
    return float(np.max(err)), err


def test_oracle_tlm_vs_fd():
    cfg, S = small_case(n=8)
    o = Oracle(cfg)
    o.set_state(0, S)
    p = params()
    nsteps = 4
    J, g = o.adjoint_tlm(nsteps, p)
    assert np.isfinite(J) and J > 0
    h = 1e-3
    # the three largest pre-factor sensitivities and the mobility scale
    ks = list(np.argsort(-np.abs(g[:NR]))[:3]) + [NR]
    for k in ks:
        step = h * (p[k] if k == NR else 1.0)
        Jp, _ = o.adjoint_tlm(nsteps, p + step * unit(k))
        Jm, _ = o.adjoint_tlm(nsteps, p - step * unit(k))
        fd = (Jp - Jm) / (2 * step)
        assert fd_ok(g[k], fd, J, step), (k, fd, g[k])
    # the mobility scale must matter in this set-up (the flux adjoint is exercised)
    assert abs(g[NR]) > 1e-8 * J


@pytest.mark.gpu
def test_adjoint_forward_parity(require_gpu):
    cfg, S = small_case()
    g = vb.Vidyut(cfg)
    o = Oracle(cfg)
    g.set_state(0, S)
    o.set_state(0, S)
    p = params()
    g.adjoint_set_params(p)
    nsteps = 6
    Jg, ug = g.adjoint_forward(nsteps, species=True)
    Jo, _, uo = o.adjoint_tlm(nsteps, p, species=True)
    assert abs(Jg - Jo) <= 1e-12 * abs(Jo)
    for s in range(uo.shape[0]):
        d = np.sqrt(np.mean((ug[s] - uo[s]) ** 2)) / np.sqrt(np.mean(uo[s] ** 2))
        assert d <= 1e-12, (s, d)
    # the state itself is untouched
    np.testing.assert_array_equal(g.get_state(0, 8), S[:8])


@pytest.mark.gpu
@pytest.mark.parametrize("hyp_order,weno", [(5, 3), (5, 1), (5, 2), (2, 3), (1, 3)])
def test_adjoint_vs_tlm(require_gpu, hyp_order, weno):
    cfg, S = small_case()
    cfg["hyp_order"] = hyp_order
    cfg["weno_scheme"] = weno
    g = vb.Vidyut(cfg)
    o = Oracle(cfg)
    g.set_state(0, S)
    o.set_state(0, S)
    p = params(1)
    g.adjoint_set_params(p)
    nsteps = 7
    Jg, gg = g.adjoint_run(nsteps, K=3)
    Jo, go = o.adjoint_tlm(nsteps, p)
    assert abs(Jg - Jo) <= 1e-12 * abs(Jo)
    worst, _ = grad_close(gg, go, 1e-9)
    assert worst <= 1e-9, worst


def periodic_walled(cfg):
    """x periodic; walls that zero the flux (IHNEUBC) on the ions' z-lo and
    the electrons' y-hi sides."""
    cfg["is_periodic"] = [1, 0, 0]
    cfg["pot_bc_lo"] = [0, 2, 1]
    cfg["pot_bc_hi"] = [0, 2, 1]
    for key in ("eden", "ion", "neutral", "eenrg"):
        cfg[f"{key}_bc_lo"] = [0, 2, 3 if key == "ion" else 2]
        cfg[f"{key}_bc_hi"] = [0, 3 if key == "eden" else 2, 2]
    return cfg


def line_case(kind):
    if kind == "2d":
        cfg = W.adjoint_config(12, prob_hi=[2e-4, 2e-4, 2e-4], dt=5e-12)
        cfg["dim"] = 2
        cfg["n_cell"] = [16, 12, 1]
        cfg["prob_hi"] = [2e-4, 1.5e-4, 1.0]
        cfg["pot_bc_lo"] = [2, 1, 2]
        cfg["pot_bc_hi"] = [2, 1, 2]
        cfg["voltage_amp_hi"] = [0.0, 20e3, 0.0]
        return cfg, W.adjoint_state(cfg, 4, efield=5e6)
    cfg, S = small_case(n=10 if kind == "periodic_walled" else 12)
    if kind == "periodic_walled":
        periodic_walled(cfg)
    return cfg, S


# The WENO face adjoint by line march (k_adj_faces_line, the default) and by
# one thread per face (VD_ADJ_FACES_LINE=0): the same derivatives summed in
# another order; and the line march against the oracle's tangent-linear
# gradient with a periodic direction and flux-zeroing walls.
@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "periodic_walled", "2d"])
def test_adjoint_face_line_march(require_gpu, monkeypatch, kind):
    cfg, S = line_case(kind)
    p = params(5)
    runs = []
    for v in ("1", "0"):
        monkeypatch.setenv("VD_ADJ_FACES_LINE", v)
        g = vb.Vidyut(cfg)
        g.set_state(0, S)
        g.adjoint_set_params(p)
        runs.append(g.adjoint_run(6, K=4))
        g.close()
    (J1, g1), (J0, g0) = runs
    assert J1 == J0
    worst, _ = grad_close(g1, g0, 1e-12)
    assert worst <= 1e-12, worst
    o = Oracle(cfg)
    o.set_state(0, S)
    Jo, go = o.adjoint_tlm(6, p)
    assert abs(J1 - Jo) <= 1e-12 * abs(Jo)
    worst, _ = grad_close(g1, go, 1e-9)
    assert worst <= 1e-9, worst


# The forward step as chemistry + one line march per direction (each face
# flux formed once, the default) against one thread per cell forming both of
# its faces (VD_ADJ_STEP_LINE=0): the same map summed in another order, for
# every flux scheme; and the gradient of the line-march map against the
# oracle's tangent-linear gradient with a periodic direction and walls.
@pytest.mark.gpu
@pytest.mark.parametrize("kind,hyp", [("box", 5), ("periodic_walled", 5), ("2d", 5),
                                      ("periodic_walled", 2), ("periodic_walled", 1)])
def test_adjoint_step_line_march(require_gpu, monkeypatch, kind, hyp):
    cfg, S = line_case(kind)
    cfg["hyp_order"] = hyp
    p = params(6)
    out = []
    for v in ("1", "0"):
        monkeypatch.setenv("VD_ADJ_STEP_LINE", v)
        g = vb.Vidyut(cfg)
        g.set_state(0, S)
        g.adjoint_set_params(p)
        J, u = g.adjoint_forward(6, species=True)
        out.append((J, u, g.adjoint_run(6, K=4)))
        g.close()
    (J1, u1, (Ja1, g1)), (J0, u0, (Ja0, g0)) = out
    assert abs(J1 - J0) <= 1e-13 * abs(J0)
    assert abs(Ja1 - J1) <= 1e-13 * abs(J1)
    for s in range(u0.shape[0]):
        d = np.sqrt(np.mean((u1[s] - u0[s]) ** 2)) / np.sqrt(np.mean(u0[s] ** 2))
        assert d <= 1e-13, (s, d)
    # the two maps differ by rounding, which the WENO weights' derivatives
    # amplify (3.4e-11 measured on the periodic walled case): the oracle
    # comparison's bound
    worst, _ = grad_close(g1, g0, 1e-9)
    assert worst <= 1e-9, worst
    o = Oracle(cfg)
    o.set_state(0, S)
    Jo, go = o.adjoint_tlm(6, p)
    assert abs(J1 - Jo) <= 1e-12 * abs(Jo)
    worst, _ = grad_close(g1, go, 1e-9)
    assert worst <= 1e-9, worst


# Lines split into segments (the launch's own choice: 8 at these sizes, and
# 3) against whole lines: the forward map's segments each form their own
# faces, so the state is the same bit for bit; the adjoint's seam cells take
# atomic adds from two segments, so the gradient agrees to rounding.
@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "periodic_walled", "2d"])
def test_adjoint_line_segments(require_gpu, monkeypatch, kind):
    cfg, S = line_case(kind)
    p = params(7)
    out = []
    for v in ("1", None, "3"):
        if v is None:
            monkeypatch.delenv("VD_ADJ_LINE_SEGMENTS", raising=False)
        else:
            monkeypatch.setenv("VD_ADJ_LINE_SEGMENTS", v)
        g = vb.Vidyut(cfg)
        g.set_state(0, S)
        g.adjoint_set_params(p)
        J, u = g.adjoint_forward(5, species=True)
        out.append((J, u, g.adjoint_run(5, K=2)))
        g.close()
    J1, u1, (_, g1) = out[0]
    for J, u, (Ja, gr) in out[1:]:
        assert J == J1 and Ja == J1
        assert np.array_equal(u, u1)
        worst, _ = grad_close(gr, g1, 1e-12)
        assert worst <= 1e-12, worst


@pytest.mark.gpu
def test_adjoint_checkpoint_intervals(require_gpu):
    cfg, S = small_case()
    g = vb.Vidyut(cfg)
    g.set_state(0, S)
    g.adjoint_set_params(params(2))
    ref = None
    for K in (1, 2, 3, 10, 25):
        J, gr = g.adjoint_run(10, K=K)
        if ref is None:
            ref = (J, gr)
        else:
            assert abs(J - ref[0]) <= 1e-13 * abs(ref[0])
            worst, _ = grad_close(gr, ref[1], 1e-12)
            assert worst <= 1e-12, (K, worst)


def fd_gradient(g, p, nsteps, ks, h):
    out = {}
    for k in ks:
        step = h * (p[k] if k == NR else 1.0)
        g.adjoint_set_params(p + step * unit(k))
        Jp = g.adjoint_forward(nsteps)
        g.adjoint_set_params(p - step * unit(k))
        Jm = g.adjoint_forward(nsteps)
        out[k] = (Jp - Jm) / (2 * step)
    g.adjoint_set_params(p)
    return out


@pytest.mark.gpu
def test_adjoint_vs_fd_small(require_gpu):
    cfg, S = small_case()
    g = vb.Vidyut(cfg)
    g.set_state(0, S)
    p = params(4)
    g.adjoint_set_params(p)
    nsteps = 10
    J, gr = g.adjoint_run(nsteps, K=4)
    h = 1e-3
    fd = fd_gradient(g, p, nsteps, range(NR + 1), h=h)
    for k in range(NR + 1):
        assert fd_ok(gr[k], fd[k], J, h * (p[k] if k == NR else 1.0)), (k, gr[k], fd[k])


def cell_difference_fd(g, p, nsteps, k, h, dV):
    """Central difference of J = sum n_e dV formed cell by cell: the final
    electron densities at p + h e_k and p - h e_k are subtracted per cell
    (exact: the two values lie within a factor 2) and the differences summed
    with math.fsum (correctly rounded).  This avoids the quantisation of a
    difference of two rounded totals (one unit in the last place of J,
    3.8e-6 at J = 2.3e10, over 2h), leaving only the per-cell rounding of
    the forward map, which cancels across cells."""
    import math

    step = h * (p[k] if k == NR else 1.0)
    g.adjoint_set_params(p + step * unit(k))
    _, up = g.adjoint_forward(nsteps, species=True)
    g.adjoint_set_params(p - step * unit(k))
    _, um = g.adjoint_forward(nsteps, species=True)
    g.adjoint_set_params(p)
    return math.fsum((up[0] - um[0]).ravel().tolist()) * dV / (2.0 * step)


@pytest.mark.gpu
def test_adjoint_c4_vs_fd(require_gpu):
    """The 128^3 workload: 50 steps at dt = 1e-12 s, checkpoints every 10;
    the four largest pre-factor sensitivities, one small one, and the
    mobility scale.

    * Central differences of J at h = 1e-6 (the step the workload states).
      Their floor is the rounding of J itself: J(p +- h) are doubles, each
      within half a unit in the last place, so the quotient is resolved to
      ulp(J) / (2h), about 1.9 at J = 2.3e10 (gradient entries are <= ~900):
      |g - fd| <= 1e-6 |fd| + ulp(J) / h.
    * Central differences formed cell by cell (cell_difference_fd) at
      h = 4e-3, 2e-3 and 1e-3, Richardson-extrapolated in pairs,
      R1 = (4 D(2e-3) - D(4e-3)) / 3 and R2 = (4 D(1e-3) - D(2e-3)) / 3
      (truncation O(h^4), ~1e-12 relative here).  The per-cell rounding
      noise of a difference grows as 1/h (6e-7 relative at h = 1e-4 on
      this workload), so the larger steps keep it near 1e-7; |R1 - R2|
      measures what remains.  Bound: |g - R2| <= 1e-6 |R2| + 2 |R1 - R2|,
      and on the four large entries that measured floor must itself be
      below 1e-6 of the entry, so that the check resolves 1e-6 relative."""
    cfg = W.adjoint_config(128)
    S = W.adjoint_state(cfg, 0)
    g = vb.Vidyut(cfg)
    g.set_state(0, S)
    p = np.zeros(NR + 1)
    p[NR] = 1.0
    g.adjoint_set_params(p)
    nsteps = 50
    J, gr = g.adjoint_run(nsteps, K=10)
    assert np.all(np.isfinite(gr)) and J > 0
    order = np.argsort(-np.abs(gr[:NR]))
    ks = list(order[:4]) + [int(order[12]), NR]
    h = 1e-6
    fd = fd_gradient(g, p, nsteps, ks, h=h)
    ulp = float(np.spacing(J))
    for k in ks:
        step = h * (p[k] if k == NR else 1.0)
        assert abs(gr[k] - fd[k]) <= 1e-6 * abs(fd[k]) + ulp / step, (k, gr[k], fd[k])
    dV = float(np.prod([(cfg["prob_hi"][d] - cfg["prob_lo"][d]) / cfg["n_cell"][d]
                        for d in range(3)]))
    for k in ks:
        d4, d2, d1 = (cell_difference_fd(g, p, nsteps, k, hh, dV) for hh in (4e-3, 2e-3, 1e-3))
        r1 = (4.0 * d2 - d4) / 3.0
        r2 = (4.0 * d1 - d2) / 3.0
        noise = 2.0 * abs(r1 - r2)
        assert abs(gr[k] - r2) <= 1e-6 * abs(r2) + noise, (k, gr[k], r1, r2)
        if k in order[:4]:
            assert noise <= 1e-6 * abs(gr[k]), (k, gr[k], r1, r2)


@pytest.mark.gpu
def test_adjoint_autograd_wrapper(require_gpu):
    """torch.autograd.Function over the C ABI (test harness only)."""
    import torch

    cfg, S = small_case()
    g = vb.Vidyut(cfg)
    g.set_state(0, S)
    nsteps = 5

    class ElectronCount(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, scale):
            p = np.concatenate([theta.detach().cpu().numpy(),
                                [float(scale.detach().cpu())]]).astype(np.float64)
            g.adjoint_set_params(p)
            J, gr = g.adjoint_run(nsteps, K=2)
            ctx.save_for_backward(torch.from_numpy(gr))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (gr,) = ctx.saved_tensors
            return gout * gr[:NR], gout * gr[NR]

    theta = torch.zeros(NR, dtype=torch.float64, requires_grad=True)
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    J = ElectronCount.apply(theta, scale)
    (2.0 * J).backward()
    p = np.zeros(NR + 1)
    p[NR] = 1.0
    g.adjoint_set_params(p)
    h = 1e-3
    fd = fd_gradient(g, p, nsteps, [NR, int(torch.argmax(theta.grad.abs()))], h=h)
    for k, ref in fd.items():
        got = float(scale.grad) if k == NR else float(theta.grad[k])
        assert fd_ok(got / 2.0, ref, float(J), h), (k, got, ref)
