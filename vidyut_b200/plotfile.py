"""AMReX plotfile writer/reader for one uniform level, and the reference's
field comparator on plotfiles.

The reference writes its state with amrex::WriteMultiLevelPlotfile
(Source/Plot.cpp:32-44): a directory holding a text ``Header`` (the
"HyperCLaw-V1.1" plotfile header: variable names, dimension, time, domain,
cell sizes, grids per level), and ``Level_0/Cell_H`` (VisMF header: boxes,
file offsets, per-box min/max) plus ``Level_0/Cell_D_00000`` (FAB data: an
ASCII FAB header line, then the box's components one after another, x
fastest, little-endian IEEE doubles).  Variable names are the reference's
(Source/Vidyut.cpp:34-74).  This module writes that layout from a state array
(ncomp, nz, ny, nx) and reads it back, so that runs of this library can be
opened with the usual AMReX tools and compared field by field
(py_utils/compare_fields_from_twoplotfiles.py:40-46).  The whole level is
written as one box.
"""
from __future__ import annotations

import os
import re

import numpy as np

PLASMA_VARS = [
    "Electron_energy", "Electron_Temp", "Potential", "Efieldx", "Efieldy", "Efieldz",
    "Electron_Jheat", "Electron_inelasticHeat", "Electron_elasticHeat", "ReducedEF",
    "SurfaceCharge", "PhotoIon_Src", "cellmask", "Ecurden_X", "Ecurden_Y", "Ecurden_Z",
    "Icurden_X", "Icurden_Y", "Icurden_Z", "Dcurden_X", "Dcurden_Y", "Dcurden_Z",
]

_FAB_REAL = "(8, (64 11 52 0 1 12 0 1023))"
_FAB_ORDER = "(8, (1 2 3 4 5 6 7 8))"


def var_names(species: list[str]) -> list[str]:
    return list(species) + PLASMA_VARS


def _box(dim, hi):
    lo = ",".join("0" for _ in range(dim))
    h = ",".join(str(x) for x in hi[:dim])
    t = ",".join("0" for _ in range(dim))
    return f"(({lo}) ({h}) ({t}))"


def write_plotfile(path: str, state: np.ndarray, names: list[str], prob_lo, prob_hi,
                   time: float = 0.0, step: int = 0, dim: int = 3) -> None:
    """Write ``state`` (ncomp, nz, ny, nx) as a single-level plotfile."""
    state = np.ascontiguousarray(state, dtype="<f8")
    ncomp = state.shape[0]
    assert len(names) == ncomp
    n = [state.shape[3], state.shape[2], state.shape[1]]
    hi = [x - 1 for x in n]
    dx = [(prob_hi[d] - prob_lo[d]) / n[d] for d in range(dim)]
    os.makedirs(os.path.join(path, "Level_0"), exist_ok=True)
    fmt = lambda v: " ".join(repr(float(x)) for x in v)  # noqa: E731
    with open(os.path.join(path, "Header"), "w") as f:
        f.write("HyperCLaw-V1.1\n")
        f.write(f"{ncomp}\n")
        for nm in names:
            f.write(nm + "\n")
        f.write(f"{dim}\n{float(time)!r}\n0\n")
        f.write(fmt(prob_lo[:dim]) + " \n")
        f.write(fmt(prob_hi[:dim]) + " \n")
        f.write("\n")                      # refinement ratios (one level: none)
        f.write(_box(dim, hi) + " \n")
        f.write(f"{step} \n")
        f.write(fmt(dx) + " \n")
        f.write("0\n0\n")                  # coordinate system, boundary width
        f.write(f"0 1 {float(time)!r}\n{step}\n")
        for d in range(dim):
            f.write(f"{float(prob_lo[d])!r} {float(prob_hi[d])!r}\n")
        f.write("Level_0/Cell\n")
    box = _box(dim, hi)
    fab_hdr = f"FAB ({_FAB_REAL},{_FAB_ORDER}){box} {ncomp}\n".encode()
    with open(os.path.join(path, "Level_0", "Cell_D_00000"), "wb") as f:
        f.write(fab_hdr)
        f.write(state.tobytes(order="C"))
    mins = state.reshape(ncomp, -1).min(axis=1)
    maxs = state.reshape(ncomp, -1).max(axis=1)
    with open(os.path.join(path, "Level_0", "Cell_H"), "w") as f:
        f.write("1\n1\n")                  # VisMF version, how
        f.write(f"{ncomp}\n0\n")           # ncomp, ngrow
        f.write(f"(1 0\n{box}\n)\n")
        f.write("1\nFabOnDisk: Cell_D_00000 0\n\n")
        f.write(f"1,{ncomp}\n" + ",".join(repr(float(x)) for x in mins) + ",\n\n")
        f.write(f"1,{ncomp}\n" + ",".join(repr(float(x)) for x in maxs) + ",\n")


def read_plotfile(path: str) -> dict:
    """Read a single-box, single-level plotfile written in the layout above."""
    with open(os.path.join(path, "Header")) as f:
        lines = f.read().splitlines()
    assert lines[0].startswith("HyperCLaw")
    ncomp = int(lines[1])
    names = lines[2:2 + ncomp]
    q = 2 + ncomp
    dim = int(lines[q])
    time = float(lines[q + 1])
    prob_lo = [float(x) for x in lines[q + 3].split()]
    prob_hi = [float(x) for x in lines[q + 4].split()]
    with open(os.path.join(path, "Level_0", "Cell_D_00000"), "rb") as f:
        raw = f.read()
    nl = raw.index(b"\n")
    hdr = raw[:nl].decode()
    m = re.search(r"\(\(([-\d,]+)\) \(([-\d,]+)\) \(([-\d,]+)\)\) (\d+)$", hdr)
    lo = [int(x) for x in m.group(1).split(",")]
    hi = [int(x) for x in m.group(2).split(",")]
    nc = int(m.group(4))
    n = [h - l + 1 for l, h in zip(lo, hi)] + [1] * (3 - dim)
    data = np.frombuffer(raw[nl + 1:], dtype="<f8").reshape(nc, n[2], n[1], n[0])
    return {"names": names, "dim": dim, "time": time, "prob_lo": prob_lo,
            "prob_hi": prob_hi, "data": data.copy()}


def compare_plotfiles(p1: str, p2: str, var1: str, var2: str | None = None):
    """Absolute and relative error of one field between two plotfiles, the
    metric of py_utils/compare_fields_from_twoplotfiles.py:40-46."""
    from .compare import field_error

    a = read_plotfile(p1)
    b = read_plotfile(p2)
    f1 = a["data"][a["names"].index(var1)]
    f2 = b["data"][b["names"].index(var2 or var1)]
    return field_error(f1, f2)
