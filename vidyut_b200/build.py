"""Build the CUDA library, one shared object per case directory.

Each case directory under ``vidyut_b200/cases/`` (the reference's per-case
Chemistry.H / UserFunctions.H / UserSources.H / Prob.H / ProbParm.H layout)
is compiled into ``vidyut_b200/lib/libvd_<case>.so`` for sm_100a, the way the
reference builds one executable per case (test/Make.vidyut).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
CASES = os.path.join(PKG, "cases")
LIBDIR = os.path.join(PKG, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-shared", "-Xcudafe", "--diag_suppress=177",
]


COMPAT = os.path.join(PKG, "compat")

# case directories outside vidyut_b200/cases (register_case)
EXTRA_CASES: dict[str, str] = {}


def cases() -> list[str]:
    return sorted(d for d in os.listdir(CASES)
                  if os.path.isfile(os.path.join(CASES, d, "Chemistry.H")))


def register_case(name: str, path: str) -> None:
    """Build case `name` from the case directory at `path` (for example a
    reference test/verification or test/models directory, compiled
    unchanged through the compatibility headers in vidyut_b200/compat)."""
    EXTRA_CASES[name] = os.path.abspath(path)


def case_dir(case: str) -> str:
    return EXTRA_CASES.get(case, os.path.join(CASES, case))


def reference_style(cdir: str) -> bool:
    """A case directory written against AMReX, as the reference's are (it
    includes AMReX headers, and keeps species names in Chemistry.cpp)."""
    if os.path.isfile(os.path.join(cdir, "Chemistry.cpp")):
        return True
    for f in os.listdir(cdir):
        if f.endswith(".H"):
            with open(os.path.join(cdir, f), errors="replace") as fh:
                if "<AMReX_" in fh.read():
                    return True
    return False


def case_flags(case: str) -> tuple[list[str], list[str]]:
    """Include flags and extra sources of one case directory: a reference
    case directory adds the compatibility headers and its Chemistry.cpp."""
    cdir = case_dir(case)
    inc = ["-I", cdir]
    extra = []
    if reference_style(cdir):
        inc += ["-I", COMPAT]
        cpp = os.path.join(cdir, "Chemistry.cpp")
        if os.path.isfile(cpp):
            extra.append(cpp)
    return inc, extra


def lib_path(case: str) -> str:
    return os.path.join(LIBDIR, f"libvd_{case}.so")


def sources() -> list[str]:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))]


def _stale(case: str) -> bool:
    out = lib_path(case)
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    cdir = case_dir(case)
    deps = sources() + [os.path.join(cdir, f) for f in os.listdir(cdir)]
    deps += [os.path.join(COMPAT, f) for f in os.listdir(COMPAT)]
    deps.append(os.path.join(ROOT, "include", "vidyut_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build_case(case: str, force: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = lib_path(case)
    if not force and not _stale(case):
        return out
    inc, srcs = case_flags(case)
    cmd = [NVCC, *NVCC_FLAGS, *(extra or []), *inc,
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           f'-DVD_CASE_NAME="{case}"',
           os.path.join(CSRC, "vd_lib.cu"), *srcs, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for case {case}:\n{r.stderr[-6000:]}")
    os.replace(out + ".tmp", out)
    return out


HOST = os.path.join(PKG, "host", "vd_run.cpp")


def host_path(case: str) -> str:
    return os.path.join(LIBDIR, f"vd_run_{case}")


def build_host(case: str, force: bool = False) -> str:
    """The C++ host driver (host/vd_run.cpp) linked against one case
    library through the C ABI only (include/vidyut_b200.h)."""
    lib = build_case(case)
    out = host_path(case)
    if (not force and os.path.exists(out) and
            os.path.getmtime(out) >= max(os.path.getmtime(HOST), os.path.getmtime(lib))):
        return out
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), HOST,
           "-L", LIBDIR, f"-lvd_{case}", "-Wl,-rpath,$ORIGIN", "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host build failed for case {case}:\n{r.stderr[-4000:]}")
    os.replace(out + ".tmp", out)
    return out


PEAK_SRC = os.path.join(PKG, "peak", "vd_fp64peak.cu")


def peak_path() -> str:
    return os.path.join(LIBDIR, "libvd_fp64peak.so")


def build_peak(force: bool = False) -> str:
    """The FP64 CUDA-core throughput probe (peak/vd_fp64peak.cu), the
    denominator of the explicit kernel's roofline."""
    os.makedirs(LIBDIR, exist_ok=True)
    out = peak_path()
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(PEAK_SRC):
        return out
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
           "-Xcompiler", "-fPIC", "-shared", PEAK_SRC, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for the FP64 probe:\n{r.stderr[-4000:]}")
    os.replace(out + ".tmp", out)
    return out


def build_all(force: bool = False) -> list[str]:
    build_peak(force)
    cs = cases()
    with ThreadPoolExecutor(max_workers=min(4, len(cs))) as ex:
        out = list(ex.map(lambda c: build_case(c, force), cs))
    for c in cs:
        build_host(c, force)
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    only = [a for a in sys.argv[1:] if not a.startswith("-")]
    for c in (only or cases()):
        print(build_case(c, force))
