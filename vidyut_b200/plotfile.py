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
written as one box; the reader also takes the many-box files an AMReX run
writes (boxes placed by their index ranges, either FAB byte order).

Checkpoints follow Vidyut::WriteCheckpointFile / ReadCheckpointFile
(Source/Plot.cpp:46-222): ``Header`` holds the title line, finest_level, the
istep, dt and t_new arrays (one entry per level, 17 significant digits) and
the BoxArray; ``Level_0/phi_H`` + ``phi_D_00000`` hold every state component
in the same VisMF layout.
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


_BOX_RE = re.compile(r"\(\(([-\d,]+)\) \(([-\d,]+)\) \(([-\d,]+)\)\)")


def _parse_box(text: str):
    m = _BOX_RE.search(text)
    lo = [int(x) for x in m.group(1).split(",")]
    hi = [int(x) for x in m.group(2).split(",")]
    return lo, hi


def _write_vismf(level_dir: str, prefix: str, state: np.ndarray, dim: int) -> None:
    """One-box VisMF MultiFab: ``<prefix>_D_00000`` (FAB header line, then the
    components x fastest, little-endian doubles) and ``<prefix>_H``."""
    ncomp = state.shape[0]
    n = [state.shape[3], state.shape[2], state.shape[1]]
    box = _box(dim, [x - 1 for x in n])
    data = f"{prefix}_D_00000"
    fab_hdr = f"FAB ({_FAB_REAL},{_FAB_ORDER}){box} {ncomp}\n".encode()
    with open(os.path.join(level_dir, data), "wb") as f:
        f.write(fab_hdr)
        f.write(np.ascontiguousarray(state, dtype="<f8").tobytes(order="C"))
    mins = state.reshape(ncomp, -1).min(axis=1)
    maxs = state.reshape(ncomp, -1).max(axis=1)
    with open(os.path.join(level_dir, f"{prefix}_H"), "w") as f:
        f.write("1\n1\n")                  # VisMF version, how
        f.write(f"{ncomp}\n0\n")           # ncomp, ngrow
        f.write(f"(1 0\n{box}\n)\n")
        f.write(f"1\nFabOnDisk: {data} 0\n\n")
        f.write(f"1,{ncomp}\n" + ",".join(repr(float(x)) for x in mins) + ",\n\n")
        f.write(f"1,{ncomp}\n" + ",".join(repr(float(x)) for x in maxs) + ",\n")


def _read_vismf(level_dir: str, prefix: str, dim: int, dom_lo, dom_hi) -> np.ndarray:
    """A VisMF MultiFab on the domain [dom_lo, dom_hi] as one array
    (ncomp, nz, ny, nx): every FAB listed in ``<prefix>_H`` read from its file
    and offset and placed at its box (ghost cells dropped)."""
    with open(os.path.join(level_dir, f"{prefix}_H")) as f:
        lines = f.read().splitlines()
    ncomp = int(lines[2])
    # ngrow: one width for every direction, or an IntVect "(gx,gy,gz)" when
    # the widths differ by direction
    gtxt = lines[3].strip()
    if gtxt.startswith("("):
        gw = [int(v) for v in gtxt.strip("()").replace(" ", "").split(",") if v]
    else:
        gw = [int(gtxt)] * 3
    gw = (gw + [0, 0, 0])[:3]
    fabs = [ln.split()[1:] for ln in lines if ln.startswith("FabOnDisk:")]
    n = [dom_hi[d] - dom_lo[d] + 1 for d in range(dim)] + [1] * (3 - dim)
    out = np.zeros((ncomp, n[2], n[1], n[0]))
    for name, off in fabs:
        with open(os.path.join(level_dir, name), "rb") as f:
            f.seek(int(off))
            hdr = f.readline().decode()
            lo, hi = _parse_box(hdr[hdr.rindex("(("):])
            nc = int(hdr.split()[-1])
            big = "(8 7 6 5 4 3 2 1)" in hdr
            m = [hi[d] - lo[d] + 1 for d in range(dim)] + [1] * (3 - dim)
            raw = f.read(8 * nc * m[0] * m[1] * m[2])
        a = np.frombuffer(raw, dtype=">f8" if big else "<f8").reshape(nc, m[2], m[1], m[0])
        g = [gw[d] for d in range(dim)] + [0] * (3 - dim)
        vlo = [lo[d] + g[d] - dom_lo[d] for d in range(dim)] + [0] * (3 - dim)
        v = a[:, g[2]:m[2] - g[2], g[1]:m[1] - g[1], g[0]:m[0] - g[0]]
        out[:, vlo[2]:vlo[2] + v.shape[1], vlo[1]:vlo[1] + v.shape[2],
            vlo[0]:vlo[0] + v.shape[3]] = v
    return out


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
    _write_vismf(os.path.join(path, "Level_0"), "Cell", state, dim)


def read_plotfile(path: str) -> dict:
    """Read a single-level plotfile (one box or many)."""
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
    lo, hi = _parse_box(lines[q + 6])
    data = _read_vismf(os.path.join(path, "Level_0"), "Cell", dim, lo, hi)
    return {"names": names, "dim": dim, "time": time, "prob_lo": prob_lo,
            "prob_hi": prob_hi, "data": data}


def compare_plotfiles(p1: str, p2: str, var1: str, var2: str | None = None):
    """Absolute and relative error of one field between two plotfiles, the
    metric of py_utils/compare_fields_from_twoplotfiles.py:40-46."""
    from .compare import field_error

    a = read_plotfile(p1)
    b = read_plotfile(p2)
    f1 = a["data"][a["names"].index(var1)]
    f2 = b["data"][b["names"].index(var2 or var1)]
    return field_error(f1, f2)


def write_checkpoint(path: str, state: np.ndarray, time: float, step: int, dt: float,
                     dim: int = 3) -> None:
    """Write a single-level checkpoint in the reference's layout."""
    n = [state.shape[3], state.shape[2], state.shape[1]]
    os.makedirs(os.path.join(path, "Level_0"), exist_ok=True)
    with open(os.path.join(path, "Header"), "w") as f:
        f.write("Checkpoint file for Vidyut\n")
        f.write("0\n")                                   # finest_level
        f.write(f"{int(step)} \n")                       # istep per level
        f.write(f"{float(dt):.17g} \n")                  # dt per level
        f.write(f"{float(time):.17g} \n")                # t_new per level
        f.write(f"(1 0\n{_box(dim, [x - 1 for x in n])}\n)\n")  # BoxArray
    _write_vismf(os.path.join(path, "Level_0"), "phi", state, dim)


def read_checkpoint(path: str) -> dict:
    """Read level 0 of a checkpoint: step, dt, time and the state array
    (ncomp, nz, ny, nx) assembled from all of its boxes."""
    with open(os.path.join(path, "Header")) as f:
        lines = f.read().splitlines()
    if not lines[0].startswith("Checkpoint file for Vidyut"):
        raise ValueError(f"{path}: not a Vidyut checkpoint")
    step = int(lines[2].split()[0])
    dt = float(lines[3].split()[0])
    time = float(lines[4].split()[0])
    # level 0's BoxArray: "(nbox 0", the boxes, ")"
    nbox = int(lines[5].strip("(").split()[0])
    boxes = [_parse_box(lines[6 + b]) for b in range(nbox)]
    dim = lines[6].count(",") // 3 + 1
    lo = [min(b[0][d] for b in boxes) for d in range(dim)]
    hi = [max(b[1][d] for b in boxes) for d in range(dim)]
    data = _read_vismf(os.path.join(path, "Level_0"), "phi", dim, lo, hi)
    return {"step": step, "dt": dt, "time": time, "dim": dim, "data": data}
