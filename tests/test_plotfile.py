"""AMReX plotfile layout (Source/Plot.cpp:32-44): round trip of a state
through the writer and reader, the reference's variable names, and the
reference comparator (py_utils/compare_fields_from_twoplotfiles.py:40-46)
on two plotfiles."""
import os

import numpy as np

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import plotfile as pf
from vidyut_b200 import workloads as W


def test_roundtrip_and_names(tmp_path):
    cfg = W.townsend_config(3, 12)
    o = Oracle(cfg)
    o.set_state(0, W.initial_state(cfg, 3))
    o.step(1)
    S = o.get_state()
    names = pf.var_names(vb.case_info("townsend")["names"])
    assert names[:3] == ["E", "ION", "N"] and names[3] == "Electron_energy"
    assert names[3 + 9] == "ReducedEF" and len(names) == S.shape[0]
    p = str(tmp_path / "plt00001")
    pf.write_plotfile(p, S, names, [0, 0, 0], [0.02, 0.02, 0.02], time=5e-13, step=1)
    hdr = open(os.path.join(p, "Header")).read().splitlines()
    assert hdr[0] == "HyperCLaw-V1.1" and int(hdr[1]) == S.shape[0]
    assert "((0,0,0) (11,11,11) (0,0,0))" in open(os.path.join(p, "Header")).read()
    r = pf.read_plotfile(p)
    assert r["names"] == names and r["dim"] == 3 and r["time"] == 5e-13
    assert np.array_equal(r["data"], S)


def test_compare_plotfiles(tmp_path):
    S = np.random.default_rng(0).uniform(1.0, 2.0, size=(3, 4, 5, 6))
    T = S.copy()
    T[1] *= 1.0 + 1e-6
    pf.write_plotfile(str(tmp_path / "a"), S, ["A", "B", "C"], [0, 0, 0], [1, 1, 1])
    pf.write_plotfile(str(tmp_path / "b"), T, ["A", "B", "C"], [0, 0, 0], [1, 1, 1])
    assert pf.compare_plotfiles(str(tmp_path / "a"), str(tmp_path / "b"), "A") == (0.0, 0.0)
    err, rel = pf.compare_plotfiles(str(tmp_path / "a"), str(tmp_path / "b"), "B")
    assert 5e-7 < rel < 2e-6


def test_reader_takes_per_direction_ghost_widths(tmp_path):
    """AMReX writes the VisMF ngrow line as an IntVect such as (2,1,0) when
    the ghost widths differ by direction; the FAB on disk then holds the
    grown box, and the reader drops each direction's own width."""
    rng = np.random.default_rng(1)
    S = rng.uniform(size=(2, 3, 4, 5))          # (ncomp, nz, ny, nx)
    p = str(tmp_path / "plt")
    pf.write_plotfile(p, S, ["A", "B"], [0, 0, 0], [1, 1, 1])
    g = (2, 1, 0)
    grown = np.full((2, 3 + 2 * g[2], 4 + 2 * g[1], 5 + 2 * g[0]), -7.0)
    grown[:, g[2]:g[2] + 3, g[1]:g[1] + 4, g[0]:g[0] + 5] = S
    lvl = os.path.join(p, "Level_0")
    box = f"(({-g[0]},{-g[1]},{-g[2]}) ({4 + g[0]},{3 + g[1]},{2 + g[2]}) (0,0,0))"
    with open(os.path.join(lvl, "Cell_D_00000"), "wb") as f:
        f.write(f"FAB (8, (64 11 52 0 1 12 0 1023))(8, (1 2 3 4 5 6 7 8)){box} 2\n".encode())
        f.write(np.ascontiguousarray(grown, dtype="<f8").tobytes())
    hdr = open(os.path.join(lvl, "Cell_H")).read().splitlines()
    hdr[3] = "(2,1,0)"
    open(os.path.join(lvl, "Cell_H"), "w").write("\n".join(hdr) + "\n")
    r = pf.read_plotfile(p)
    assert np.array_equal(r["data"], S)
