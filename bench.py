"""Benchmark: cell-steps/s of the per-timestep species-and-field update.

Workload: the 3-D Townsend discharge on a uniform 256^3 grid (2 cm cube,
20 kV across z, five seeded Gaussian blobs, WENO5-Z drift, dt = 5e-13 s),
two transported species plus a background gas, FP64 state.  A "step" is one
full coarse step (Poisson multigrid solve, field, reactions + drift fluxes,
implicit diffusion multigrid solve per species, write-back).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vidyut_b200|reference]

One process per GPU (torchrun for N > 1); the path does not shard, so N > 1
runs N independent replicas ("weak" scaling; barrier and max-over-ranks
device time).  `--impl reference` times the CPU restatement of the reference
step (the reference, an AMReX application, cannot be built here) on the host
cores, rank 0 only, on a 96^3 sample of the same workload per step.

Timing: device time of the K steps from CUDA events on the library's stream;
inputs (3.4 GB of state) exceed the 126 MB L2 between steps.
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


def make(n: int, precision: int, device: int):
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n)
    cfg["mg_precision"] = precision
    cfg["device"] = device
    return cfg


def cpu_sample(steps: int, n: int = 128) -> dict:
    """CPU restatement of the reference step, timed on the host cores."""
    from oracle.oracle import Oracle
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 0))
    t0 = time.perf_counter()
    o.step(steps)
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n ** 3 * steps / el, "unit": "cell-steps/s", "cores": cores,
            "kind": "port", "seconds": el,
            "sample": f"{steps} step(s) of the same workload on a {n}^3 grid "
                      f"(oracle/vd_oracle.cpp, g++ -O3 -fopenmp, {cores} threads)"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    n = 96
    from oracle.oracle import Oracle
    from vidyut_b200 import workloads as W
    cfg = W.townsend_config(3, n)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 0))
    o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    v = n ** 3 * args.steps / el
    line = {
        "metric": "cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "townsend_3d (two-species Townsend discharge, WENO5-Z, "
                               "dt 5e-13 s)", "grid": [n, n, n], "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"each step one step of the workload on a {n}^3 grid "
                                   "(CPU restatement of the reference step; the reference "
                                   "itself needs AMReX, absent here)"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    (forward, recompute, backward), host synchronised on both sides."""
    import torch
    import vidyut_b200 as vb
    from vidyut_b200 import workloads as W

    cfg = W.adjoint_config(n, device=device)
    g = vb.Vidyut(cfg)
    g.set_state(0, W.adjoint_state(cfg, 0))
    g.adjoint_run(5, K=5)  # warm-up
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    g.adjoint_forward(nsteps)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    J, grad = g.adjoint_run(nsteps, K=K)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    g.close()
    fwd = dist_max(dist, t1 - t0)
    run = dist_max(dist, t2 - t1)
    return {"workload": f"LMEA 8 species / 30 reactions, {n}^3, {nsteps} explicit flux+source "
                        f"steps at dt 1e-12 s, checkpoints every {K}, objective sum n_e dV, "
                        "31 parameters",
            "forward_ms": 1e3 * fwd, "adjoint_run_ms": 1e3 * run,
            "adjoint_over_forward": run / fwd,
            "forward_cell_steps_per_s": n ** 3 * nsteps / fwd,
            "objective": J, "grad_norm": float(np.linalg.norm(grad))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vidyut_b200")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
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
    clk = clocks.stop()
    ms_p = dist_max(dist, st_p.gpu_ms)

    # roofline of the dominant kernel (fine-level Poisson RB sweep)
    peak, peak_kind = load_peaks()
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
            "pass": f"second run of the {args.steps} timed steps with per-launch events "
                    f"({ms_p / args.steps:.3f} ms/step under the events)",
            "traffic": (traffic or {}).get("bytes_per_launch") if traffic else None,
            "traffic_note": (traffic or {}).get("note") if traffic else None}

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

    # FP32-refined multigrid form on the same workload
    cfg32 = make(n, vb.VD_MG_FP32_REFINED, local)
    g32 = vb.Vidyut(cfg32)
    g32.set_state(0, state)
    g32.step(args.warmup)
    st32, _, _ = timed(g32, args.steps, dist, 0)
    ms32 = dist_max(dist, st32.gpu_ms)
    value32 = replica_value(world, ncell, args.steps, ms32)
    # Poisson error of the refined form against the FP64 form, same state
    ga, gb = vb.Vidyut(make(n, vb.VD_MG_FP64, local)), g32
    ga.set_state(0, state)
    gb.set_state(0, state)
    ga.solve_potential(0.0)
    gb.solve_potential(0.0)
    pa = ga.get_state(info["pot_id"], 1)
    pb = gb.get_state(info["pot_id"], 1)
    perr = float(np.linalg.norm(pb - pa) / np.linalg.norm(pa))
    ga.close()
    gb.close()

    adj = None if args.no_adjoint else adjoint_leg(local, dist)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_sample(8, 128)
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
            "cpu_baseline": cpu,
            "solver": {"poisson_vcycles_per_step": st.poisson_iterations / args.steps,
                       "species_vcycles_per_step": st.species_iterations / args.steps},
            "fp32_refined": {"value": value32, "ms_per_step": ms32 / args.steps,
                             "speedup_vs_fp64": value32 / value,
                             "poisson_rel_err_vs_fp64": perr,
                             "poisson_vcycles_per_step": st32.poisson_iterations / args.steps},
            "adjoint": adj,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
