"""ctypes loader of the CPU oracle -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker (or the timed CPU baseline) of the CUDA library.  The
interface mirrors vidyut_b200.Vidyut so a parity test reads the same on both
sides.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import vidyut_b200 as vb  # noqa: E402
from oracle import build as obuild  # noqa: E402

_LIBS: dict[str, C.CDLL] = {}


def load(case: str) -> C.CDLL:
    if case in _LIBS:
        return _LIBS[case]
    path = obuild.build_case(case)
    lib = C.CDLL(path)
    P = C.c_void_p
    sig = {
        "vdo_create": [C.POINTER(vb.vd_config), C.POINTER(C.c_void_p)],
        "vdo_destroy": [P],
        "vdo_init_domain": [P, C.c_char_p],
        "vdo_set_probinit": [P, C.c_char_p],
        "vdo_set_state": [P, C.c_int, C.c_int, P],
        "vdo_get_state": [P, C.c_int, C.c_int, P],
        "vdo_set_time": [P, C.c_double, C.c_int],
        "vdo_step": [P, C.c_int, C.POINTER(vb.vd_step_stats)],
        "vdo_poisson_solve": [P, C.c_double, C.POINTER(vb.vd_solve_stats)],
        "vdo_explicit_rhs": [P, C.c_double, P],
        "vdo_implicit_diffusion": [P, C.c_int, C.c_double, P, C.POINTER(vb.vd_solve_stats)],
        "vdo_implicit_diffusion_chunk": [P, C.c_int, C.c_int, C.c_double, P,
                                         C.POINTER(vb.vd_solve_stats)],
        "vdo_adjoint_tlm": [P, C.c_int, C.POINTER(C.c_double), C.c_int,
                            C.POINTER(C.c_double), C.POINTER(C.c_double), P],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    _LIBS[case] = lib
    return lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class Oracle:
    def __init__(self, cfg: "vb.Config"):
        self.cfg = cfg
        self.lib = load(cfg.case)
        self.info = vb.case_info(cfg.case)
        self.ctx = C.c_void_p()
        assert self.lib.vdo_create(C.byref(cfg.c), C.byref(self.ctx)) == 0
        c = cfg.c
        self.shape = tuple(c.n_cell[d] if d < c.dim else 1 for d in range(3))
        self.ncell = int(np.prod(self.shape))

    def close(self):
        if self.ctx:
            self.lib.vdo_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_domain(self, prob_inputs: str = ""):
        self.lib.vdo_init_domain(self.ctx, prob_inputs.encode())

    def set_probinit(self, prob_inputs: str = ""):
        self.lib.vdo_set_probinit(self.ctx, prob_inputs.encode())

    def set_state(self, comp: int, data: np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.float64)
        self.lib.vdo_set_state(self.ctx, comp, a.size // self.ncell, _ptr(a))

    def get_state(self, comp: int = 0, ncomp: int | None = None) -> np.ndarray:
        if ncomp is None:
            ncomp = self.info["nvar"] - comp
        out = np.empty((ncomp, self.shape[2], self.shape[1], self.shape[0]))
        self.lib.vdo_get_state(self.ctx, comp, ncomp, _ptr(out))
        return out

    def set_time(self, t: float, step: int = 0):
        self.lib.vdo_set_time(self.ctx, t, step)

    def step(self, nsteps: int = 1) -> "vb.vd_step_stats":
        st = vb.vd_step_stats()
        self.lib.vdo_step(self.ctx, nsteps, C.byref(st))
        return st

    def solve_potential(self, time: float = 0.0, allow_unconverged: bool = True) -> "vb.vd_solve_stats":
        st = vb.vd_solve_stats()
        self.lib.vdo_poisson_solve(self.ctx, time, C.byref(st))
        return st

    def explicit_rhs(self, time: float = 0.0) -> np.ndarray:
        ns = self.info["num_species"]
        out = np.empty((ns + 1, self.shape[2], self.shape[1], self.shape[0]))
        self.lib.vdo_explicit_rhs(self.ctx, time, _ptr(out))
        return out

    def implicit_solve_scalar(self, specid: int, expl_src: np.ndarray, time: float = 0.0,
                              allow_unconverged: bool = True):
        a = np.ascontiguousarray(expl_src, dtype=np.float64)
        st = vb.vd_solve_stats()
        self.lib.vdo_implicit_diffusion(self.ctx, specid, time, _ptr(a), C.byref(st))
        return st

    def implicit_solve_chunk(self, startspec: int, numspec: int, expl_src: np.ndarray,
                             time: float = 0.0, allow_unconverged: bool = True):
        a = np.ascontiguousarray(expl_src, dtype=np.float64)
        st = vb.vd_solve_stats()
        self.lib.vdo_implicit_diffusion_chunk(self.ctx, startspec, numspec, time, _ptr(a),
                                              C.byref(st))
        return st

    def adjoint_tlm(self, nsteps: int, params, species: bool = False):
        """Objective and gradient of the library's adjoint forward map by an
        FP64 tangent-linear pass (all parameter directions at once)."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        g = np.zeros(p.size)
        J = C.c_double()
        out = None
        if species:
            nt = self.info["num_species"] - int(self.cfg.c.num_bg_species)
            out = np.empty((nt, self.shape[2], self.shape[1], self.shape[0]))
        dp = C.POINTER(C.c_double)
        st = self.lib.vdo_adjoint_tlm(self.ctx, nsteps, p.ctypes.data_as(dp), p.size,
                                      C.byref(J), g.ctypes.data_as(dp),
                                      _ptr(out) if out is not None else None)
        if st != 0:
            raise RuntimeError(f"vdo_adjoint_tlm failed with status {st}")
        return (J.value, g, out) if species else (J.value, g)
