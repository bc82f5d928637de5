"""vidyut_b200 -- B200-native per-timestep species-and-field update of Vidyut3d.

Python host binding of the C ABI in ``include/vidyut_b200.h``.  The compute
path is the CUDA library ``vidyut_b200/lib/libvd_<case>.so`` (one build per
case directory, like the reference's one executable per case); this module
only loads it with ctypes and mirrors the reference's run-time interface:

* :class:`Config` holds the reference's ParmParse parameters
  (``vidyut.*``, ``amr.n_cell``, ``geometry.*``) with the reference's defaults
  and accepts inputs-file text (:meth:`Config.from_inputs`);
* :class:`Vidyut` is one uniform-level run: ``init_domain`` (amrex_probinit +
  initdomaindata), ``step`` (Vidyut::Evolve's step body), and the sub-stages
  ``solve_potential``, ``explicit_rhs``, ``implicit_solve_scalar``.

There is no CPU fallback: constructing :class:`Vidyut` without a loadable
CUDA library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(PKG, "lib")

VD_MAX_SPECIES = 64
VD_MG_FP64 = 0
VD_MG_FP32_REFINED = 1

STATUS = {0: "VD_OK", 1: "VD_ERR_INVALID_ARG", 2: "VD_ERR_CUDA", 3: "VD_ERR_NOT_CONVERGED",
          4: "VD_ERR_UNSUPPORTED", 5: "VD_ERR_OOM", 6: "VD_ERR_NONFINITE"}

_I3 = C.c_int * 3
_D3 = C.c_double * 3


class vd_config(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n_cell", _I3), ("prob_lo", _D3), ("prob_hi", _D3),
        ("is_periodic", _I3), ("dt", C.c_double), ("num_timestep_correctors", C.c_int),
        ("electron_poisson_coupling", C.c_int), ("electron_poisson_maxiters", C.c_int),
        ("adaptive_dt", C.c_int), ("advective_cfl", C.c_double), ("diffusive_cfl", C.c_double),
        ("dielectric_cfl", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("adaptive_dt_delay", C.c_double), ("dt_stretch", C.c_double),
        ("hyp_order", C.c_int), ("weno_scheme", C.c_int),
        ("do_reactions", C.c_int), ("do_transport", C.c_int), ("do_spacechrg", C.c_int),
        ("elecenergy_solve", C.c_int), ("using_LFA", C.c_int), ("floor_jh", C.c_int),
        ("bound_specden", C.c_int), ("do_bg_reactions", C.c_int),
        ("user_defined_potential", C.c_int), ("user_defined_species", C.c_int),
        ("user_defined_vel", C.c_int),
        ("min_species_density", C.c_double), ("min_electron_density", C.c_double),
        ("min_electron_temp", C.c_double), ("gas_temperature", C.c_double),
        ("gas_pressure", C.c_double),
        ("pot_bc_lo", _I3), ("pot_bc_hi", _I3), ("eden_bc_lo", _I3), ("eden_bc_hi", _I3),
        ("eenrg_bc_lo", _I3), ("eenrg_bc_hi", _I3), ("ion_bc_lo", _I3), ("ion_bc_hi", _I3),
        ("neutral_bc_lo", _I3), ("neutral_bc_hi", _I3),
        ("voltage_profile", C.c_int), ("voltage_amp_lo", _D3), ("voltage_amp_hi", _D3),
        ("voltage_freq", C.c_double), ("voltage_dur", C.c_double),
        ("voltage_center", C.c_double),
        ("linsolve_reltol", C.c_double), ("linsolve_abstol", C.c_double),
        ("linsolve_bot_reltol", C.c_double), ("linsolve_bot_abstol", C.c_double),
        ("linsolve_num_pre_smooth", C.c_int), ("linsolve_num_post_smooth", C.c_int),
        ("linsolve_num_final_smooth", C.c_int), ("linsolve_num_bottom_smooth", C.c_int),
        ("linsolve_maxiter", C.c_int), ("linsolve_max_coarsening_level", C.c_int),
        ("potential_scale", C.c_double), ("elecenergy_scale", C.c_double),
        ("time_scale", C.c_double), ("species_scale", C.c_double * VD_MAX_SPECIES),
        ("num_bg_species", C.c_int), ("bg_species_ids", C.c_int * VD_MAX_SPECIES),
        ("mg_precision", C.c_int), ("mg_inner_cycles", C.c_int),
        ("poisson_warm_start", C.c_int), ("device", C.c_int),
        ("multicompsolves", C.c_int), ("comp_ion_chunks", C.c_int),
        ("comp_neutral_chunks", C.c_int),
    ]


class vd_case_info_t(C.Structure):
    _fields_ = [
        ("num_species", C.c_int), ("nvar", C.c_int), ("e_id", C.c_int),
        ("een_id", C.c_int), ("etemp_id", C.c_int), ("pot_id", C.c_int), ("efx_id", C.c_int),
        ("ref_id", C.c_int), ("ejh_id", C.c_int), ("eih_id", C.c_int), ("cmask_id", C.c_int),
        ("charge", C.c_int * VD_MAX_SPECIES), ("names", (C.c_char * 16) * VD_MAX_SPECIES),
        ("case_name", C.c_char * 64),
    ]


class vd_solve_stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("converged", C.c_int),
                ("initial_residual", C.c_double), ("final_residual", C.c_double)]


class vd_step_stats(C.Structure):
    _fields_ = [("steps", C.c_int), ("poisson_iterations", C.c_int),
                ("species_iterations", C.c_int), ("not_converged", C.c_int),
                ("max_poisson_final_residual", C.c_double), ("time", C.c_double),
                ("gpu_ms", C.c_double), ("dt", C.c_double), ("dt_edrift", C.c_double),
                ("dt_ediff", C.c_double), ("dt_diel_relax", C.c_double),
                ("poisson_refinements", C.c_int)]


EXPORTS = [
    "vd_config_init", "vd_config_set", "vd_case_info", "vd_create", "vd_destroy",
    "vd_init_domain", "vd_set_state", "vd_get_state", "vd_set_time", "vd_get_time",
    "vd_set_dt", "vd_get_dt",
    "vd_step", "vd_poisson_solve", "vd_explicit_rhs", "vd_implicit_diffusion",
    "vd_check_state", "vd_launch_count", "vd_profile_kernel", "vd_profile_read",
    "vd_last_error", "vd_poisson_solve_noalloc", "vd_adjoint_num_params",
    "vd_implicit_diffusion_chunk",
    "vd_adjoint_set_params", "vd_adjoint_forward", "vd_adjoint_run",
]

VD_ADJ_OBJ_ELECTRONS = 0

VD_PROF_NONE = 0
VD_PROF_POISSON_SMOOTH = 1
VD_PROF_EXPLICIT = 2
VD_PROF_POISSON_SMOOTH32 = 3
VD_PROF_EFIELD = 4
VD_PROF_POISSON_RHS = 5
VD_PROF_SPECIES_RHS = 6


class VidyutError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        super().__init__(f"{where}: {STATUS.get(status, status)} {msg}".strip())
        self.status = status


def lib_path(case: str) -> str:
    return os.path.join(LIBDIR, f"libvd_{case}.so")


_LIBS: dict[str, C.CDLL] = {}


def load(case: str) -> C.CDLL:
    """Load (building on first use if absent) the CUDA library of `case`."""
    if case in _LIBS:
        return _LIBS[case]
    from . import build
    path = build.build_case(case)  # no-op unless missing or older than its sources
    lib = C.CDLL(path)
    P = C.c_void_p
    sig = {
        "vd_config_init": [C.POINTER(vd_config)],
        "vd_config_set": [C.POINTER(vd_config), C.c_char_p, C.c_char_p],
        "vd_case_info": [C.POINTER(vd_case_info_t)],
        "vd_create": [C.POINTER(vd_config), C.POINTER(C.c_void_p)],
        "vd_destroy": [P],
        "vd_init_domain": [P, C.c_char_p],
        "vd_set_state": [P, C.c_int, C.c_int, P, C.c_int],
        "vd_get_state": [P, C.c_int, C.c_int, P, C.c_int],
        "vd_set_time": [P, C.c_double, C.c_int],
        "vd_get_time": [P, C.POINTER(C.c_double), C.POINTER(C.c_int)],
        "vd_set_dt": [P, C.c_double],
        "vd_get_dt": [P, C.POINTER(C.c_double)],
        "vd_step": [P, C.c_int, C.POINTER(vd_step_stats)],
        "vd_poisson_solve": [P, C.c_double, C.POINTER(vd_solve_stats)],
        "vd_explicit_rhs": [P, C.c_double, P, C.c_int],
        "vd_implicit_diffusion": [P, C.c_int, C.c_double, P, C.c_int, C.POINTER(vd_solve_stats)],
        "vd_implicit_diffusion_chunk": [P, C.c_int, C.c_int, C.c_double, P, C.c_int,
                                        C.POINTER(vd_solve_stats)],
        "vd_check_state": [P, C.POINTER(C.c_longlong)],
        "vd_launch_count": [P, C.POINTER(C.c_longlong)],
        "vd_profile_kernel": [P, C.c_int],
        "vd_profile_read": [P, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                            C.POINTER(C.c_double)],
        "vd_last_error": [P, C.c_char_p, C.c_int],
        "vd_poisson_solve_noalloc": [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double), P, P,
                                     C.c_double, C.c_double, C.c_int,
                                     C.POINTER(vd_solve_stats), C.c_char_p, C.c_int],
        "vd_adjoint_num_params": [P, C.POINTER(C.c_int)],
        "vd_adjoint_set_params": [P, C.POINTER(C.c_double), C.c_int],
        "vd_adjoint_forward": [P, C.c_int, C.c_int, C.POINTER(C.c_double), P],
        "vd_adjoint_run": [P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                           C.POINTER(C.c_double), C.c_int],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    _LIBS[case] = lib
    return lib


def case_info(case: str) -> dict:
    lib = load(case)
    info = vd_case_info_t()
    _check(lib.vd_case_info(C.byref(info)), "vd_case_info")
    ns = info.num_species
    return {
        "num_species": ns, "nvar": info.nvar, "e_id": info.e_id, "een_id": info.een_id,
        "etemp_id": info.etemp_id, "pot_id": info.pot_id, "efx_id": info.efx_id,
        "ref_id": info.ref_id, "ejh_id": info.ejh_id, "eih_id": info.eih_id,
        "cmask_id": info.cmask_id, "charge": list(info.charge[:ns]),
        "names": [info.names[i].value.decode() for i in range(ns)],
        "case": info.case_name.decode(),
    }


def _check(st: int, where: str, lib=None, ctx=None):
    if st != 0:
        msg = ""
        if lib is not None:
            buf = C.create_string_buffer(512)
            lib.vd_last_error(ctx, buf, 512)
            msg = buf.value.decode(errors="replace")
        raise VidyutError(st, where, msg)


class Config:
    """Run parameters with the reference's defaults (Source/Vidyut.H:250-400)."""

    def __init__(self, case: str, **kw):
        self.case = case
        self._lib = load(case)
        self.c = vd_config()
        _check(self._lib.vd_config_init(C.byref(self.c)), "vd_config_init")
        for k, v in kw.items():
            self[k] = v

    def set(self, key: str, value) -> "Config":
        """Set by inputs-file name ("vidyut.hyp_order", "amr.n_cell", ...)."""
        if isinstance(value, (list, tuple, np.ndarray)):
            value = " ".join(str(x) for x in value)
        st = self._lib.vd_config_set(C.byref(self.c), key.encode(), str(value).encode())
        _check(st, f"vd_config_set({key})")
        return self

    def __setitem__(self, name, value):
        if "." in name:
            self.set(name, value)
            return
        cur = getattr(self.c, name)
        if isinstance(cur, (int, float)):
            setattr(self.c, name, value)
        else:
            for i, x in enumerate(value):
                cur[i] = x

    def __getitem__(self, name):
        v = getattr(self.c, name)
        return v if isinstance(v, (int, float)) else list(v)

    @classmethod
    def from_inputs(cls, case: str, text: str, **kw) -> "Config":
        """Parse reference inputs-file text (unknown keys are ignored)."""
        cfg = cls(case, **kw)
        for line in text.splitlines():
            line = line.split("#", 1)[0]
            if "=" not in line:
                continue
            k, v = (s.strip() for s in line.split("=", 1))
            if k == "amr.n_cell" and "dim" not in kw:
                # the reference's dimension is a build switch; its inputs
                # files give as many n_cell entries as it has dimensions
                cfg["dim"] = 2 if len(v.split()) == 2 else 3
            try:
                cfg.set(k, v)
            except VidyutError:
                pass
        return cfg


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Vidyut:
    """One single-level run on one GPU, driven through the C ABI."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.lib = cfg._lib
        self.info = case_info(cfg.case)
        self.ctx = C.c_void_p()
        st = self.lib.vd_create(C.byref(cfg.c), C.byref(self.ctx))
        _check(st, "vd_create", self.lib, None)
        c = cfg.c
        self.dim = c.dim
        self.shape = tuple(c.n_cell[d] if d < c.dim else 1 for d in range(3))
        self.ncell = int(np.prod(self.shape))

    # -- lifecycle
    def close(self):
        if self.ctx:
            self.lib.vd_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, st, where):
        _check(st, where, self.lib, self.ctx)

    # -- state (arrays are (ncomp, nz, ny, nx) or flat, x fastest)
    def init_domain(self, prob_inputs: str = ""):
        self._chk(self.lib.vd_init_domain(self.ctx, prob_inputs.encode()), "vd_init_domain")

    def set_state(self, comp: int, data: np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.float64)
        ncomp = a.size // self.ncell
        assert ncomp * self.ncell == a.size
        self._chk(self.lib.vd_set_state(self.ctx, comp, ncomp, _ptr(a), 0), "vd_set_state")

    def get_state(self, comp: int = 0, ncomp: int | None = None) -> np.ndarray:
        if ncomp is None:
            ncomp = self.info["nvar"] - comp
        out = np.empty((ncomp, self.shape[2], self.shape[1], self.shape[0]))
        self._chk(self.lib.vd_get_state(self.ctx, comp, ncomp, _ptr(out), 0), "vd_get_state")
        return out

    def set_time(self, t: float, step: int = 0):
        self._chk(self.lib.vd_set_time(self.ctx, t, step), "vd_set_time")

    def time(self) -> tuple[float, int]:
        t = C.c_double()
        s = C.c_int()
        self._chk(self.lib.vd_get_time(self.ctx, C.byref(t), C.byref(s)), "vd_get_time")
        return t.value, s.value

    def set_dt(self, dt: float):
        self._chk(self.lib.vd_set_dt(self.ctx, dt), "vd_set_dt")

    def dt(self) -> float:
        v = C.c_double()
        self._chk(self.lib.vd_get_dt(self.ctx, C.byref(v)), "vd_get_dt")
        return v.value

    # -- stepping and sub-stages
    def step(self, nsteps: int = 1, allow_unconverged: bool = False) -> vd_step_stats:
        st = vd_step_stats()
        r = self.lib.vd_step(self.ctx, nsteps, C.byref(st))
        if not (allow_unconverged and r == 3):
            self._chk(r, "vd_step")
        return st

    def solve_potential(self, time: float = 0.0, allow_unconverged: bool = False) -> vd_solve_stats:
        st = vd_solve_stats()
        r = self.lib.vd_poisson_solve(self.ctx, time, C.byref(st))
        if not (allow_unconverged and r == 3):
            self._chk(r, "vd_poisson_solve")
        return st

    def explicit_rhs(self, time: float = 0.0) -> np.ndarray:
        ns = self.info["num_species"]
        out = np.empty((ns + 1, self.shape[2], self.shape[1], self.shape[0]))
        self._chk(self.lib.vd_explicit_rhs(self.ctx, time, _ptr(out), 0), "vd_explicit_rhs")
        return out

    def implicit_solve_scalar(self, specid: int, expl_src: np.ndarray,
                              time: float = 0.0, allow_unconverged: bool = False) -> vd_solve_stats:
        st = vd_solve_stats()
        if getattr(expl_src, "is_cuda", False):
            # a contiguous FP64 CUDA tensor on the context's device: no copy
            assert expl_src.is_contiguous() and str(expl_src.dtype) == "torch.float64"
            r = self.lib.vd_implicit_diffusion(self.ctx, specid, time,
                                               C.c_void_p(expl_src.data_ptr()), 1, C.byref(st))
        else:
            a = np.ascontiguousarray(expl_src, dtype=np.float64)
            r = self.lib.vd_implicit_diffusion(self.ctx, specid, time, _ptr(a), 0, C.byref(st))
        if not (allow_unconverged and r == 3):
            self._chk(r, "vd_implicit_diffusion")
        return st

    def implicit_solve_chunk(self, startspec: int, numspec: int, expl_src: np.ndarray,
                             time: float = 0.0, allow_unconverged: bool = False) -> vd_solve_stats:
        """Species [startspec, startspec + numspec) solved together
        (vd_implicit_diffusion_chunk)."""
        a = np.ascontiguousarray(expl_src, dtype=np.float64)
        st = vd_solve_stats()
        r = self.lib.vd_implicit_diffusion_chunk(self.ctx, startspec, numspec, time, _ptr(a), 0,
                                                 C.byref(st))
        if not (allow_unconverged and r == 3):
            self._chk(r, "vd_implicit_diffusion_chunk")
        return st

    def check_state(self) -> int:
        n = C.c_longlong()
        r = self.lib.vd_check_state(self.ctx, C.byref(n))
        if r not in (0, 6):
            self._chk(r, "vd_check_state")
        return n.value

    def profile_kernel(self, kernel_id: int):
        self._chk(self.lib.vd_profile_kernel(self.ctx, kernel_id), "vd_profile_kernel")

    def profile_read(self) -> tuple[int, float, float]:
        n = C.c_longlong()
        ms = C.c_double()
        b = C.c_double()
        self._chk(self.lib.vd_profile_read(self.ctx, C.byref(n), C.byref(ms), C.byref(b)),
                  "vd_profile_read")
        return n.value, ms.value, b.value

    def write_plotfile(self, path: str) -> None:
        """The full state as an AMReX plotfile (Source/Plot.cpp:32-44 layout)."""
        from .plotfile import var_names, write_plotfile
        c = self.cfg.c
        t, step = self.time()
        write_plotfile(path, self.get_state(), var_names(self.info["names"]),
                       list(c.prob_lo), list(c.prob_hi), t, step, self.dim)

    def write_checkpoint(self, path: str) -> None:
        """State, step count, dt and time in the reference's checkpoint layout
        (Vidyut::WriteCheckpointFile, Source/Plot.cpp:46-132)."""
        from .plotfile import write_checkpoint
        t, step = self.time()
        write_checkpoint(path, self.get_state(), t, step, self.dt(), self.dim)

    def restart(self, path: str) -> None:
        """Continue from a checkpoint (Vidyut::ReadCheckpointFile,
        Source/Plot.cpp:134-222): state, time, step count and dt."""
        from .plotfile import read_checkpoint
        ck = read_checkpoint(path)
        data = ck["data"]
        if data.shape[1:] != (self.shape[2], self.shape[1], self.shape[0]):
            raise ValueError(f"checkpoint grid {data.shape[1:]} does not match the run")
        if data.shape[0] != self.info["nvar"]:
            raise ValueError(f"checkpoint has {data.shape[0]} components, the case {self.info['nvar']}")
        self.set_state(0, data)
        self.set_time(ck["time"], ck["step"])
        self.set_dt(ck["dt"])

    # -- discrete adjoint of explicit flux + source steps (no reference counterpart)
    def adjoint_num_params(self) -> int:
        n = C.c_int()
        self._chk(self.lib.vd_adjoint_num_params(self.ctx, C.byref(n)), "vd_adjoint_num_params")
        return n.value

    def adjoint_set_params(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._chk(self.lib.vd_adjoint_set_params(
            self.ctx, p.ctypes.data_as(C.POINTER(C.c_double)), p.size), "vd_adjoint_set_params")

    def adjoint_forward(self, nsteps: int, species: bool = False,
                        objective: int = VD_ADJ_OBJ_ELECTRONS):
        """Objective after `nsteps` steps of the adjoint's forward map (and the
        final transported species, (nt, nz, ny, nx), when `species`)."""
        J = C.c_double()
        out = None
        if species:
            nt = self.info["num_species"] - int(self.cfg.c.num_bg_species)
            out = np.empty((nt, self.shape[2], self.shape[1], self.shape[0]))
        self._chk(self.lib.vd_adjoint_forward(self.ctx, nsteps, objective, C.byref(J),
                                              _ptr(out) if out is not None else None),
                  "vd_adjoint_forward")
        return (J.value, out) if species else J.value

    def adjoint_run(self, nsteps: int, K: int, objective: int = VD_ADJ_OBJ_ELECTRONS):
        """(objective, gradient) by the checkpointed backward sweep."""
        n = self.adjoint_num_params()
        g = np.zeros(n)
        J = C.c_double()
        self._chk(self.lib.vd_adjoint_run(self.ctx, nsteps, K, objective, C.byref(J),
                                          g.ctypes.data_as(C.POINTER(C.c_double)), n),
                  "vd_adjoint_run")
        return J.value, g

    def launch_count(self) -> int:
        n = C.c_longlong()
        self._chk(self.lib.vd_launch_count(self.ctx, C.byref(n)), "vd_launch_count")
        return n.value
