"""Benchmark: cell-steps/s of the per-timestep species-and-field update.

Workload (the headline): the 3-D Townsend discharge on a uniform 256^3 grid
(2 cm cube, 20 kV across z, five seeded Gaussian blobs, WENO5-Z drift,
dt = 5e-13 s), two transported species plus a background gas, FP64 state,
in the plain form (the reference's scheme: FP64 multigrid, zero initial
guess of the potential).  A "step" is one full coarse step (Poisson
multigrid solve, field, reactions + drift fluxes, implicit diffusion
multigrid solve per species, write-back).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vidyut_b200|reference]

One process per GPU (torchrun for N > 1); the path does not shard, so N > 1
runs N independent replicas ("weak" scaling; barrier and max-over-ranks
device time).  `--impl reference` times the CPU restatement of the reference
step (the reference, an AMReX application, cannot be built here) on the host
cores, rank 0 only, on the same 256^3 workload.

Timing: device time of the K steps from CUDA events on the library's stream;
inputs (3.4 GB of state) exceed the 126 MB L2 between steps.  Extra legs on
the same line: the other multigrid forms of the same step (FP64 and FP32
refinement, zero or warm initial guess) with their Poisson error against an
FP64 solve converged to 1e-13; the step's own roofline from its algorithmic
bytes; the 512^3 mixed-precision Poisson + implicit-diffusion workload; the
192^3 LMEA step with the electron-energy equation; the 2-D 256^2 run of 100
steps; the 128^3 discrete adjoint.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

HBM_FALLBACK_GBS = 6650.0


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def load_traffic():
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu
    summary (profiles/roofline_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def fp64_peak_gflops() -> float | None:
    """FP64 FMA throughput of the current GPU (vidyut_b200/peak)."""
    import ctypes
    from vidyut_b200 import build
    try:
        lib = ctypes.CDLL(build.build_peak())
        lib.vd_fp64_peak_gflops.restype = ctypes.c_double
        lib.vd_fp64_peak_gflops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        v = lib.vd_fp64_peak_gflops(8, 20000, 5)
        return v if v > 0 else None
    except Exception:
        return None


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


class Clocks:
    """nvidia-smi sampler of SM clocks and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend: str | None = None):
    """One process per GPU; the replicas exchange nothing but a barrier and
    the max-over-ranks time (NCCL on GPUs, gloo for the CPU tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or os.environ.get("VD_DIST_BACKEND", "nccl")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return world, rank, local, dist


def dist_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, ncell: int, steps: int, max_ms: float) -> float:
    """Whole-job cell-steps/s of `world` replicas timed by the slowest."""
    return world * ncell * steps / (max_ms / 1e3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def make(n: int, precision: int, device: int, warm: int = 0, **kw):
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n, **kw)
    cfg["mg_precision"] = precision
    cfg["poisson_warm_start"] = warm
    cfg["device"] = device
    return cfg


def cpu_sample(n: int = 256, steps: int = 2) -> dict:
    """CPU restatement of the reference step, timed on the host cores on the
    headline workload itself (a bounded number of steps), plus the 2-D
    256^2 run of 100 steps in full."""
    from oracle.oracle import Oracle
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 0))
    t0 = time.perf_counter()
    o.step(steps)
    el = time.perf_counter() - t0
    o.close()
    c2 = W.townsend_config(2, 256)
    o2 = Oracle(c2)
    o2.set_state(0, W.initial_state(c2, 0))
    t1 = time.perf_counter()
    o2.step(100)
    el2 = time.perf_counter() - t1
    o2.close()
    cores = host_threads()
    return {"value": n ** 3 * steps / el, "unit": "cell-steps/s", "cores": cores,
            "cpu": cpu_model(), "kind": "port", "seconds": el,
            "sample": f"{steps} step(s) of the same workload at {n}^3 from the same initial "
                      f"state (oracle/vd_oracle.cpp, g++ -O3 -fopenmp, {cores} threads)",
            "townsend_2d_256": {"value": 256 * 256 * 100 / el2, "unit": "cell-steps/s",
                                "seconds": el2,
                                "sample": "2-D 256^2, 100 steps at dt 1e-12 s, in full"}}


# Wall-clock budget of the reference arm's timed steps (a 256^3 step of the
# CPU restatement takes 10-25 s on the host cores): the arm times K steps or
# as many as fit in the budget, whichever is fewer, so that a run with the
# GPU arm's K ends within a few minutes.
REF_BUDGET_S = 90.0


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference step on the
    host cores, on the headline workload (256^3): W untimed steps (at most
    3), then K timed steps or as many as REF_BUDGET_S allows."""
    if rank != 0:
        return
    n = args.n
    from oracle.oracle import Oracle
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 0))
    warm = min(args.warmup, 3)
    o.step(warm)
    done = 0
    t0 = time.perf_counter()
    while done < args.steps:
        o.step(1)
        done += 1
        if time.perf_counter() - t0 > REF_BUDGET_S:
            break
    el = time.perf_counter() - t0
    cores = host_threads()
    v = n ** 3 * done / el
    line = {
        "metric": "cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": done, "steps_requested": args.steps, "warmup": warm,
        "ms_per_step": 1e3 * el / done, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "townsend_3d: two-species Townsend discharge + background "
                               "gas, 2 cm cube, 20 kV across z, 5 seeded blobs, WENO5-Z, "
                               "dt 5e-13 s, FP64 multigrid (reference scheme)",
                   "grid": [n, n, n], "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores, "cpu": cpu_model(),
                         "kind": "port",
                         "sample": f"{done} timed steps of the workload at {n}^3 (of "
                                   f"{args.steps} requested, within {REF_BUDGET_S:.0f} s) after "
                                   f"{warm} untimed (CPU restatement of the reference step; the "
                                   "reference itself needs AMReX, absent here)"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Algorithmic bytes per cell of the step's kernels: one read of each
# distinct input array and one write of each output per launch (FP64 8 B,
# FP32 4 B), the per-kernel table of the path's measurement plan.
B_POISSON_RHS = 24.0
B_VCYCLE64 = (4 * 24 + 17 + 17) * 8.0 / 7.0      # constant coefficients, V(2,2)
B_VCYCLE32 = B_VCYCLE64 / 2.0
B_VCYCLE64_VAR = (4 * 32 + 17 + 17) * 8.0 / 7.0  # face coefficients (species)
B_REFINE = 40.0                                  # FP64 residual 20 + update 20
B_EFIELD = 64.0
B_EXPLICIT = 72.0
B_SPECIES_SETUP = 24.0
B_FINALIZE = 16.0


def step_bytes(pv: float, sv: float, nspec: int, refines: float = 0.0,
               fp32: bool = False, warm: bool = False) -> float:
    """B_step per cell for the Townsend step: RHS, n_V potential V-cycles,
    E field, explicit sources, per species set-up + its V-cycles, finalize;
    the refined form's FP64 refinement passes; a warm start's extra norm
    pass over the zero-guess residual (16 B)."""
    b = B_POISSON_RHS + pv * (B_VCYCLE32 if fp32 else B_VCYCLE64) + B_EFIELD + B_EXPLICIT
    b += nspec * B_SPECIES_SETUP + sv * B_VCYCLE64_VAR + nspec * B_FINALIZE
    b += refines * B_REFINE + (16.0 if warm else 0.0)
    return b


def timed(g, steps: int, dist, prof_id: int):
    import torch
    g.profile_kernel(prof_id)
    barrier(dist)
    torch.cuda.synchronize()
    l0 = g.launch_count()
    st = g.step(steps)
    torch.cuda.synchronize()
    barrier(dist)
    l1 = g.launch_count()
    prof = g.profile_read()
    g.profile_kernel(0)
    return st, l1 - l0, prof


def adjoint_leg(device: int, dist, n: int = 128, nsteps: int = 50, K: int = 10) -> dict:
    """Gradient of the electron count after 50 explicit LMEA steps at 128^3
    (30 log pre-factors + electron mobility scale), checkpoints every 10:
    device time of one forward-only pass and of one checkpointed adjoint run
    (forward, recompute, backward), host synchronised on both sides.  The
    warm-up run has the timed run's shape, so its checkpoint slots are
    allocated before the timed region."""
    import torch
    import vidyut_b200 as vb
    from vidyut_b200 import workloads as W

    cfg = W.adjoint_config(n, device=device)
    g = vb.Vidyut(cfg)
    g.set_state(0, W.adjoint_state(cfg, 0))
    g.adjoint_forward(nsteps)  # warm-up
    g.adjoint_run(nsteps, K=K)
    torch.cuda.synchronize()
    barrier(dist)
    clocks = Clocks(device)
    clocks.start()
    t0 = time.perf_counter()
    g.adjoint_forward(nsteps)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    J, grad = g.adjoint_run(nsteps, K=K)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    clk = clocks.stop()
    g.close()
    fwd = dist_max(dist, t1 - t0)
    run = dist_max(dist, t2 - t1)
    return {"workload": f"LMEA 8 species / 30 reactions, {n}^3, {nsteps} explicit flux+source "
                        f"steps at dt 1e-12 s, checkpoints every {K}, objective sum n_e dV, "
                        "31 parameters",
            "forward_ms": 1e3 * fwd, "adjoint_run_ms": 1e3 * run,
            "adjoint_over_forward": run / fwd,
            "forward_cell_steps_per_s": n ** 3 * nsteps / fwd,
            "objective": J, "grad_norm": float(np.linalg.norm(grad)), "clocks": clk}


def forms_leg(n: int, state, device: int, warmup: int, steps: int, dist, ref_ms: float) -> dict:
    """The other multigrid forms of the headline step: FP64 or FP32
    V-cycles (the FP32 ones inside FP64 iterative refinement), potential
    started from zero (the reference) or from the last potential with the
    zero-guess stopping target.  Each is timed like the headline (device
    time of K steps after W warm-up steps) and its Poisson error is measured
    on one solve from the state after 5 steps of the plain form, against an
    FP64 solve of the same state converged to 1e-13 (RMS difference over the
    mean magnitude)."""
    import vidyut_b200 as vb
    pid = vb.case_info("townsend")["pot_id"]
    g = vb.Vidyut(make(n, vb.VD_MG_FP64, device))
    g.set_state(0, state)
    g.step(5)
    s5 = g.get_state()
    g.close()
    g = vb.Vidyut(make(n, vb.VD_MG_FP64, device, linsolve_reltol=1e-13, linsolve_abstol=0.0))
    g.set_state(0, s5)
    g.solve_potential(0.0)
    ref = g.get_state(pid, 1)
    g.close()
    out = {}
    for name, prec, warm in (("fp64", vb.VD_MG_FP64, 0), ("fp64_warm", vb.VD_MG_FP64, 1),
                             ("fp32_refined", vb.VD_MG_FP32_REFINED, 0),
                             ("fp32_refined_warm", vb.VD_MG_FP32_REFINED, 1)):
        g = vb.Vidyut(make(n, prec, device, warm))
        g.set_state(0, s5)
        sol = g.solve_potential(0.0)
        phi = g.get_state(pid, 1)
        err = float(np.sqrt(np.mean((phi - ref) ** 2)) / np.mean(np.abs(ref)))
        g.set_state(0, state)
        g.step(warmup)
        st, _, _ = timed(g, steps, dist, 0)
        g.close()
        ms = dist_max(dist, st.gpu_ms) / steps
        pv, sv = st.poisson_iterations / steps, st.species_iterations / steps
        refs = st.poisson_refinements / steps
        out[name] = {"ms_per_step": ms, "speedup_vs_plain_fp64": ref_ms / ms,
                     "poisson_vcycles_per_step": pv, "species_vcycles_per_step": sv,
                     "poisson_refinements_per_step": refs,
                     "poisson_rel_err_vs_fp64_1e-13": err,
                     "poisson_solve_vcycles_on_error_state": sol.iterations,
                     "step_bytes_per_cell": step_bytes(pv, sv, 2, refs,
                                                       prec == vb.VD_MG_FP32_REFINED, warm == 1)}
    return out


def step_roofline(ms_per_step: float, ncell: int, bytes_per_cell: float, peak: float,
                  peak_kind: str) -> dict:
    ach = ncell * bytes_per_cell / (ms_per_step / 1e3) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_kind": peak_kind, "bytes_per_cell": bytes_per_cell,
            "note": "algorithmic bytes of the whole step (per-kernel table, measured V-cycle "
                    "counts) over its device time"}


def mgsolve_leg(device: int, n: int = 512, reps: int = 3) -> dict:
    """The 512^3 mixed-precision Poisson + implicit-diffusion workload: the
    potential solve and the ion's implicit-diffusion solve in the FP64 form
    and the FP32-refined form (FP32 V(2,2) cycles, 7 levels, inside FP64
    refinement to the reference's 1e-10 relative residual), host-timed
    around each synchronous solve (tens of ms each), best of `reps` after
    one warm-up; error of each form against the FP64 form at 1e-13."""
    import torch
    import vidyut_b200 as vb
    from vidyut_b200 import workloads as W
    pid = vb.case_info("mgsolve")["pot_id"]
    # explicit sources on the device (zero: pure implicit diffusion), so the
    # timed diffusion solve holds no host copy
    expl = torch.zeros((3, n, n, n), dtype=torch.float64, device=f"cuda:{device}")
    res = {}
    ref = {}
    # the FP64 reference: solved to the rounding floor (rel 1e-14 is out of
    # FP64's reach for this right-hand side; 60 V-cycles, status ignored)
    for name, kw in (("tight", dict(linsolve_reltol=1e-14, linsolve_abstol=0.0,
                                    linsolve_maxiter=60)),
                     ("fp64", dict(mg_precision=vb.VD_MG_FP64)),
                     ("fp32_refined", dict(mg_precision=vb.VD_MG_FP32_REFINED))):
        cfg = W.mgsolve_config(n, device=device, **kw)
        g = vb.Vidyut(cfg)
        W.mgsolve_load(g, cfg, 0)
        times_p, times_d = [], []
        for r in range(1 if name == "tight" else reps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sp = g.solve_potential(0.0, allow_unconverged=name == "tight")
            t1 = time.perf_counter()
            if r == 0:
                phi = g.get_state(pid, 1)
                ion0 = g.get_state(1, 1)
            g.set_state(1, ion0)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            sd = g.implicit_solve_scalar(1, expl, 0.0, allow_unconverged=name == "tight")
            t3 = time.perf_counter()
            if r == 0:
                ion = g.get_state(1, 1)
            g.set_state(1, ion0)
            if r > 0:
                times_p.append(t1 - t0)
                times_d.append(t3 - t2)
        g.close()
        if name == "tight":
            ref = {"phi": phi, "ion": ion}
            res["fp64_reference_residual_ratio"] = sp.final_residual / sp.initial_residual
            continue
        ep = float(np.sqrt(np.mean((phi - ref["phi"]) ** 2)) / np.mean(np.abs(ref["phi"])))
        ed = float(np.sqrt(np.mean((ion - ref["ion"]) ** 2)) / np.mean(np.abs(ref["ion"])))
        res[name] = {"poisson_ms": 1e3 * min(times_p), "poisson_vcycles": sp.iterations,
                     "poisson_refinements": sp.refinements, "poisson_rel_err": ep,
                     "diffusion_ms": 1e3 * min(times_d), "diffusion_vcycles": sd.iterations,
                     "diffusion_rel_err": ed,
                     "poisson_bytes_per_cell": sp.iterations * (B_VCYCLE32 if name != "fp64"
                                                                else B_VCYCLE64)
                     + sp.refinements * B_REFINE}
    res["poisson_speedup_fp32_refined"] = res["fp64"]["poisson_ms"] / res["fp32_refined"]["poisson_ms"]
    res["workload"] = (f"{n}^3 unit cube, 8 seeded +-1e16 m^-3 Gaussians of net charge + 1e-3 "
                       "white noise, Dirichlet z / Neumann x-y; ion diffusivity log-uniform "
                       "1e-6-1e-1 m^2/s cell by cell, dt 1e-11 s; rel tol 1e-10")
    return res


def steps_leg(cfg, state, warmup: int, steps: int) -> dict:
    import vidyut_b200 as vb
    g = vb.Vidyut(cfg)
    g.set_state(0, state)
    g.step(warmup)
    st = g.step(steps)
    g.close()
    nc = int(np.prod([cfg["n_cell"][d] for d in range(cfg["dim"])]))
    return {"ms_per_step": st.gpu_ms / steps, "cell_steps_per_s": nc * steps / (st.gpu_ms / 1e3),
            "poisson_vcycles_per_step": st.poisson_iterations / steps,
            "species_vcycles_per_step": st.species_iterations / steps, "steps": steps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vidyut_b200")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the other multigrid forms")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 512^3 solver, 192^3 LMEA and 2-D legs")
    ap.add_argument("--lean", action="store_true",
                    help="timed FP64 leg only (no e2e, FP32 or CPU legs): profiling runs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local, dist = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    import vidyut_b200 as vb
    from vidyut_b200 import workloads as W

    torch.cuda.set_device(local)
    n = args.n
    ncell = n ** 3
    cfg = make(n, vb.VD_MG_FP64, local)
    state = W.initial_state(cfg, 0)
    g = vb.Vidyut(cfg)
    g.set_state(0, state)
    g.step(args.warmup)
    clocks = Clocks(local)
    clocks.start()
    st, launches, _ = timed(g, args.steps, dist, 0)
    ms = dist_max(dist, st.gpu_ms)
    value = replica_value(world, ncell, args.steps, ms)
    # roofline pass: the same K steps again with CUDA events around every
    # fine-level Poisson sweep.  Separate from the pass above because an
    # event between two launches stops the second from overlapping the
    # first one's tail (programmatic dependent launch), which costs ~5 %
    # of the step.
    st_p, _, prof = timed(g, args.steps, dist, vb.VD_PROF_POISSON_SMOOTH)
    # and once more with events around every explicit-source launch
    _, _, prof_x = timed(g, args.steps, dist, vb.VD_PROF_EXPLICIT)
    clk = clocks.stop()
    ms_p = dist_max(dist, st_p.gpu_ms)

    # roofline of the dominant kernel (fine-level Poisson RB sweep)
    peak, peak_kind = load_peaks()

    # the step's other HBM-bound kernels, each timed live on its own pass
    # (20 steps) with events around its launches
    kernels_live = {}
    for kname, pid in (("k_efield2", vb.VD_PROF_EFIELD),
                       ("k_poisson_rhs", vb.VD_PROF_POISSON_RHS),
                       ("k_species_rhs", vb.VD_PROF_SPECIES_RHS)):
        _, _, (nk, kms, kbytes) = timed(g, min(args.steps, 20), dist, pid)
        if nk:
            ks = (kms / nk) / 1e3
            kernels_live[kname] = {"avg_launch_us": ks * 1e6, "launches_timed": nk,
                                   "algorithmic_bytes_per_launch": kbytes,
                                   "achieved_gbs": kbytes / ks / 1e9,
                                   "frac": kbytes / ks / 1e9 / peak, "peak_kind": peak_kind}
    nl, pms, pbytes = prof
    avg_s = (pms / nl) / 1e3 if nl else float("nan")
    achieved = pbytes / avg_s / 1e9 if nl else None
    traffic = load_traffic()
    roof = {"kernel": "k_mg_sweep3v<double> (Poisson fine-level red-black colour sweep, "
                      "12 B/cell: other colour of x, this colour of f, write this colour)",
            "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": pbytes, "launches_timed": nl,
            "avg_launch_us": avg_s * 1e6 if nl else None,
            "pass": f"second run of the {args.steps} timed steps with per-launch events; "
                    "launches that returned at once on the stop flag (cycles enqueued past "
                    "convergence) left out "
                    f"({ms_p / args.steps:.3f} ms/step under the events)",
            "traffic": (traffic or {}).get("bytes_per_launch") if traffic else None,
            "traffic_note": (traffic or {}).get("note") if traffic else None}

    # the explicit kernel is FP64-arithmetic bound: its roofline is the FP64
    # FLOP count per launch (ncu, committed under profiles/) over its
    # per-launch device time, against the FP64 throughput measured here
    fp64_peak = fp64_peak_gflops()
    # vd_profile_kernel brackets the whole explicit stage of a step: one
    # launch per transported component (two here), so a timed region holds
    # that many launches' FP64 work
    nx_l, xms, xbytes = prof_x
    x_avg_s = (xms / nx_l) / 1e3 if nx_l else float("nan")
    n_tr = (g.info["num_species"] - int(cfg.c.num_bg_species)
            + (1 if cfg.c.elecenergy_solve else 0))
    xflops1 = (traffic or {}).get("explicit_fp64_flops_per_launch")
    xflops = xflops1 * n_tr if xflops1 else None
    roof_explicit = {
        "kernel": "k_explicit_stream (fused reactions + WENO5-Z drift flux + divergence, one "
                  "transported component per launch)",
        "bound": "fp64", "unit": "GFLOP/s",
        "timed_region": f"the explicit stage of a step: {n_tr} launches (one per transported "
                        "component)",
        "avg_region_us": x_avg_s * 1e6 if nx_l else None,
        "regions_timed": nx_l,
        "flops_per_launch": xflops1, "flops_per_region": xflops,
        "achieved": (xflops / x_avg_s / 1e9) if (xflops and nx_l) else None,
        "peak": fp64_peak, "peak_kind": "measured (vd_fp64_peak_gflops: FP64 FMA chains)",
        "frac": (xflops / x_avg_s / 1e9 / fp64_peak) if (xflops and nx_l and fp64_peak) else None,
        "hbm_achieved_gbs": xbytes / x_avg_s / 1e9 if nx_l else None,
        "hbm_frac": (xbytes / x_avg_s / 1e9 / peak) if nx_l else None,
        "algorithmic_bytes_per_region": xbytes,
        "flops_note": (traffic or {}).get("explicit_note")}

    if args.lean:
        if rank == 0:
            print(json.dumps({"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s",
                              "n_gpus": world, "steps": args.steps, "ms_per_step": ms / args.steps,
                              "lean": True, "grid": [n, n, n], "roofline": roof}), flush=True)
        g.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    # end to end through the C ABI with pinned host buffers: state in,
    # K steps, species + potential out, all inside the timed region
    info = g.info
    nin = info["etemp_id"] + 1  # species, electron energy, electron temperature
    h_in = torch.empty((nin,) + state.shape[1:], dtype=torch.float64, pin_memory=True).numpy()
    h_in[:] = state[:nin]
    h_cm = torch.empty(state.shape[1:], dtype=torch.float64, pin_memory=True).numpy()
    h_cm[:] = state[info["cmask_id"]]
    nout = info["pot_id"] + 1
    h_out = torch.empty((nout,) + state.shape[1:], dtype=torch.float64, pin_memory=True).numpy()
    import ctypes
    barrier(dist)
    t0 = time.perf_counter()
    g.set_state(0, h_in)
    g.set_state(info["cmask_id"], h_cm)
    g.step(args.steps)
    r = g.lib.vd_get_state(g.ctx, 0, nout, ctypes.c_void_p(h_out.ctypes.data), 0)
    assert r == 0
    e2e_s = dist_max(dist, time.perf_counter() - t0)
    e2e = {"value": world * ncell * args.steps / e2e_s, "unit": "cell-steps/s",
           "h2d_bytes_per_step": (h_in.nbytes + h_cm.nbytes) / args.steps,
           "d2h_bytes_per_step": h_out.nbytes / args.steps,
           "note": f"vd_set_state (pinned host) + vd_step({args.steps}) + vd_get_state, "
                   "wall clock"}
    g.close()

    # the other multigrid forms of the same step
    forms = None if args.no_forms else forms_leg(n, state, local, args.warmup, args.steps, dist,
                                                 ms / args.steps)
    solver_legs = {}
    if not args.no_extra:
        from vidyut_b200 import workloads as W
        solver_legs["mgsolve_512"] = mgsolve_leg(local)
        c2 = W.lmea_config(192, device=local)
        solver_legs["lmea_192"] = steps_leg(c2, W.lmea_state(c2, 0), 2, 5)
        solver_legs["lmea_192"]["workload"] = (
            "LMEA 8 species / 30 reactions + electron-energy equation, 192^3, dt 1e-12 s, "
            "FP64 plain form")
        c0 = W.townsend_config(2, 256, device=local)
        solver_legs["townsend_2d_256"] = steps_leg(c0, W.initial_state(c0, 0), 3, 100)
        solver_legs["townsend_2d_256"]["workload"] = "2-D 256^2 Townsend, 100 steps at dt 1e-12 s"

    adj = None if args.no_adjoint else adjoint_leg(local, dist)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_sample(n, 2)
        pv, sv = st.poisson_iterations / args.steps, st.species_iterations / args.steps
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "townsend_3d: two-species Townsend discharge + background "
                                   "gas, 2 cm cube, 20 kV across z, 5 seeded blobs, WENO5-Z, "
                                   "dt 5e-13 s, FP64 multigrid (reference scheme)",
                       "grid": [n, n, n], "parallelism": "replicas" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (3.4 GB state)"},
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": roof,
            "roofline_explicit": roof_explicit,
            "kernels_live": kernels_live or None,
            "step_roofline": step_roofline(ms / args.steps, ncell, step_bytes(pv, sv, 2),
                                           peak, peak_kind),
            "cpu_baseline": cpu,
            "solver": {"poisson_vcycles_per_step": pv, "species_vcycles_per_step": sv},
            "forms": forms,
            "solver_workloads": solver_legs or None,
            "adjoint": adj,
        }
        if forms:
            for k, f in forms.items():
                f["step_roofline_frac"] = step_roofline(f["ms_per_step"], ncell,
                                                        f["step_bytes_per_cell"], peak,
                                                        peak_kind)["frac"]
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
