"""Checkpoint/restart in the reference's layout (Vidyut::WriteCheckpointFile /
ReadCheckpointFile, Source/Plot.cpp:46-222).

CPU: the Header lines (title, finest_level, istep, dt, t_new at 17
significant digits, BoxArray) and a bit-exact round trip of the state; a
checkpoint written as many boxes, in both FAB byte orders and with ghost
cells, as an AMReX run writes it, assembles into the same array.  GPU: a run
restarted from a checkpoint continues exactly as the uninterrupted run
(state, time, step count and the adaptive dt it stretches)."""
import os

import numpy as np
import pytest

import vidyut_b200 as vb
from vidyut_b200 import plotfile as pf
from vidyut_b200 import workloads as W


def seeded_state(shape=(25, 6, 10, 8), seed=1):
    return np.random.default_rng(seed).normal(size=shape)


def test_header_layout_and_roundtrip(tmp_path):
    S = seeded_state()
    p = str(tmp_path / "chk00007")
    t, dt = 7 * 5e-13 + 1e-25, 5e-13 * (1 + 2 ** -40)
    pf.write_checkpoint(p, S, time=t, step=7, dt=dt)
    hdr = open(os.path.join(p, "Header")).read().splitlines()
    assert hdr[0] == "Checkpoint file for Vidyut"
    assert hdr[1] == "0"
    assert hdr[2] == "7 "
    # std::ostream with precision(17): 17 significant digits, enough to
    # restore the double exactly
    assert hdr[3] == "%.17g " % dt and float(hdr[3]) == dt
    assert hdr[4] == "%.17g " % t and float(hdr[4]) == t
    assert hdr[5:8] == ["(1 0", "((0,0,0) (7,9,5) (0,0,0))", ")"]
    assert os.path.exists(os.path.join(p, "Level_0", "phi_H"))
    ck = pf.read_checkpoint(p)
    assert ck["step"] == 7 and ck["dim"] == 3
    assert ck["dt"] == dt and ck["time"] == t
    assert np.array_equal(ck["data"], S)


def write_many_boxes(path, S, ngrow=1):
    """A 3-D checkpoint of S split into 2 x 2 boxes in x and y, each FAB with
    `ngrow` ghost layers, the second box big-endian, two data files."""
    nc, nz, ny, nx = S.shape
    os.makedirs(os.path.join(path, "Level_0"), exist_ok=True)
    xs = [(0, nx // 2 - 1), (nx // 2, nx - 1)]
    ys = [(0, ny // 2 - 1), (ny // 2, ny - 1)]
    boxes = [(x, y) for y in ys for x in xs]
    g = ngrow
    pad = np.pad(S, ((0, 0), (g, g), (g, g), (g, g)), constant_values=-7.0)
    fabs = []
    files = {"phi_D_00000": b"", "phi_D_00001": b""}
    for b, ((x0, x1), (y0, y1)) in enumerate(boxes):
        lo, hi = (x0 - g, y0 - g, -g), (x1 + g, y1 + g, nz - 1 + g)
        a = pad[:, lo[2] + g:hi[2] + g + 1, lo[1] + g:hi[1] + g + 1, lo[0] + g:hi[0] + g + 1]
        order = "(8, (8 7 6 5 4 3 2 1))" if b == 1 else "(8, (1 2 3 4 5 6 7 8))"
        box = f"(({lo[0]},{lo[1]},{lo[2]}) ({hi[0]},{hi[1]},{hi[2]}) (0,0,0))"
        hdr = f"FAB ((8, (64 11 52 0 1 12 0 1023)),{order}){box} {nc}\n".encode()
        raw = np.ascontiguousarray(a, dtype=">f8" if b == 1 else "<f8").tobytes()
        name = f"phi_D_0000{b // 2}"
        fabs.append((name, len(files[name])))
        files[name] += hdr + raw
    for name, data in files.items():
        open(os.path.join(path, "Level_0", name), "wb").write(data)
    with open(os.path.join(path, "Level_0", "phi_H"), "w") as f:
        f.write(f"1\n1\n{nc}\n{g}\n({len(boxes)} 0\n")
        for (x0, x1), (y0, y1) in boxes:
            f.write(f"(({x0},{y0},0) ({x1},{y1},{nz - 1}) (0,0,0))\n")
        f.write(f")\n{len(fabs)}\n")
        for name, off in fabs:
            f.write(f"FabOnDisk: {name} {off}\n")
    with open(os.path.join(path, "Header"), "w") as f:
        f.write("Checkpoint file for Vidyut\n0\n12 \n1e-12 \n1.2e-11 \n")
        f.write(f"({len(boxes)} 0\n")
        for (x0, x1), (y0, y1) in boxes:
            f.write(f"(({x0},{y0},0) ({x1},{y1},{nz - 1}) (0,0,0))\n")
        f.write(")\n")


def test_many_box_checkpoint_assembles(tmp_path):
    S = seeded_state((25, 4, 6, 8), seed=2)
    p = str(tmp_path / "chk00012")
    write_many_boxes(p, S)
    ck = pf.read_checkpoint(p)
    assert ck["step"] == 12 and ck["dt"] == 1e-12 and ck["time"] == 1.2e-11
    assert np.array_equal(ck["data"], S)


@pytest.mark.gpu
def test_restart_continues_exactly(require_gpu, tmp_path):
    cfg = W.townsend_config(3, 32)
    cfg["adaptive_dt"] = 1
    cfg["dt_stretch"] = 1.3
    S0 = W.initial_state(cfg, 8)
    a = vb.Vidyut(cfg)
    a.set_state(0, S0)
    a.step(2)
    p = str(tmp_path / "chk00002")
    a.write_checkpoint(p)
    t_ck, dt_ck = a.time()[0], a.dt()
    a.step(2)
    b = vb.Vidyut(cfg)
    b.restart(p)
    assert b.time() == (t_ck, 2) and b.dt() == dt_ck
    sb = b.step(2)
    ta, na = a.time()
    tb, nb = b.time()
    assert na == nb == 4 and ta == tb
    assert a.dt() == b.dt() == sb.dt
    assert np.array_equal(a.get_state(), b.get_state())
