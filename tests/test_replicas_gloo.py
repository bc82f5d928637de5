"""The multi-GPU form is replicas only (the single-level step has no
exchange step that does not need a halo per smoothing sweep): bench.py runs
one independent replica per rank and reduces only the time.  This checks
that host logic with two gloo ranks on the CPU: rendezvous on 127.0.0.1,
max-over-ranks, whole-job value, and that the CPU oracle run by each rank
gives identical replica results."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    from oracle.oracle import Oracle
    from vidyut_b200 import workloads as W

    w, r, _, dist = bench.dist_setup("gloo")
    cfg = W.townsend_config(2, 16)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 0))
    o.step(2)
    ne = o.get_state(0, 1)
    mx = bench.dist_max(dist, float(rank + 1))
    bench.barrier(dist)
    out[rank] = (w, mx, bench.replica_value(w, 256, 2, mx * 1e3), float(ne.sum()))
    dist.destroy_process_group()


def test_two_gloo_replicas():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    a, b = out[0], out[1]
    assert a[0] == b[0] == 2
    assert a[1] == b[1] == 2.0            # max over ranks of (rank + 1)
    assert a[2] == 2 * 256 * 2 / 2.0      # whole-job value from the slowest rank
    assert a[3] == b[3] and np.isfinite(a[3])
