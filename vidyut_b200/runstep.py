"""Run the benchmark workload for an external profiler (ncu and the like).

    python -m vidyut_b200.runstep [--n 256] [--warmup 3] [--steps 1] [--fp32] [--warm]
    python -m vidyut_b200.runstep --n 208 --solve           # one field solve
    python -m vidyut_b200.runstep --n 192 --solve --explicit  # + explicit sources
    python -m vidyut_b200.runstep --lmea --n 192 --steps 1     # the 8-species LMEA step
    python -m vidyut_b200.runstep --adjoint --n 128 --steps 50 # the discrete adjoint

The workload is the two-species Townsend discharge of ``bench.py``
(``workloads.townsend_config(3, n)``, seeded initial state 0).  With
``--steps`` the last line reports the launches and the device time of the
timed steps, so a launch list can be cut to exactly those launches.
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--fp32", action="store_true", help="FP32-refined multigrid form")
    ap.add_argument("--warm", action="store_true",
                    help="start each potential solve from the last potential")
    ap.add_argument("--inner", type=int, default=0, help="FP32 V-cycles per refinement pass")
    ap.add_argument("--solve", action="store_true", help="one field solve instead of steps")
    ap.add_argument("--explicit", action="store_true", help="with --solve: explicit sources too")
    ap.add_argument("--lmea", action="store_true",
                    help="the 8-species LMEA workload with the electron-energy equation "
                         "(workloads.lmea_*) instead of the Townsend one")
    ap.add_argument("--adjoint", action="store_true",
                    help="the discrete-adjoint workload (workloads.adjoint_*): one warm-up "
                         "and one timed checkpointed adjoint run of --steps explicit steps, "
                         "K = 10")
    ap.add_argument("--mgsolve", action="store_true",
                    help="the solver workload (workloads.mgsolve_*): one warm-up and one "
                         "timed potential solve")
    a = ap.parse_args()

    import vidyut_b200 as vb
    from vidyut_b200 import workloads as W

    if a.adjoint:
        import time
        cfg = W.adjoint_config(a.n)
        g = vb.Vidyut(cfg)
        g.set_state(0, W.adjoint_state(cfg, 0))
        g.adjoint_run(a.steps, K=10)  # warm-up of the timed shape: slots allocated
        l0 = g.launch_count()
        t0 = time.perf_counter()
        J, grad = g.adjoint_run(a.steps, K=10)
        el = time.perf_counter() - t0
        print(f"timed adjoint run of {a.steps} steps: {g.launch_count() - l0} launches, "
              f"{1e3 * el:.3f} ms, J {J:.6e}")
        g.close()
        return
    if a.mgsolve:
        import time
        cfg = W.mgsolve_config(a.n)
        if a.fp32:
            cfg["mg_precision"] = vb.VD_MG_FP32_REFINED
        if a.inner > 0:
            cfg["mg_inner_cycles"] = a.inner
        g = vb.Vidyut(cfg)
        W.mgsolve_load(g, cfg, 0)
        g.solve_potential(0.0)
        l0 = g.launch_count()
        t0 = time.perf_counter()
        st = g.solve_potential(0.0)
        el = time.perf_counter() - t0
        print(f"timed solve: {g.launch_count() - l0} launches, {1e3 * el:.3f} ms, "
              f"V-cycles {st.iterations}, refinements {st.refinements}")
        g.close()
        return
    cfg = W.lmea_config(a.n) if a.lmea else W.townsend_config(3, a.n)
    if a.fp32:
        cfg["mg_precision"] = vb.VD_MG_FP32_REFINED
    if a.warm:
        cfg["poisson_warm_start"] = 1
    if a.inner > 0:
        cfg["mg_inner_cycles"] = a.inner
    g = vb.Vidyut(cfg)
    g.set_state(0, W.lmea_state(cfg, 0) if a.lmea else W.initial_state(cfg, 0))
    if a.solve:
        st = g.solve_potential(0.0)
        if a.explicit:
            g.explicit_rhs(0.0)
        print(f"field solve: {st.iterations} V-cycles, converged {st.converged}")
    else:
        g.step(a.warmup)
        l0 = g.launch_count()
        st = g.step(a.steps)
        print(f"timed steps {a.steps}: {g.launch_count() - l0} launches, "
              f"{st.gpu_ms:.3f} ms device time, poisson V-cycles {st.poisson_iterations}, "
              f"species V-cycles {st.species_iterations}")
    g.close()


if __name__ == "__main__":
    main()
