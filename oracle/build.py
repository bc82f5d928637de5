"""Build recipe of the CPU oracle (test infrastructure only).

Compiles ``oracle/vd_oracle.cpp`` once per case directory into
``oracle/lib/liboracle_<case>.so`` with g++ -O3 -fopenmp.  The reference
itself (an AMReX application whose AMReX submodule is empty in the
reference checkout) cannot be compiled here, so there is no ``oracle/_ref``
build; the oracle is a restatement of the reference's algorithm.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CASES = os.path.join(ROOT, "vidyut_b200", "cases")
CSRC = os.path.join(ROOT, "vidyut_b200", "csrc")
LIBDIR = os.path.join(HERE, "lib")
def _cxx() -> str:
    if os.environ.get("VD_ORACLE_CXX"):
        return os.environ["VD_ORACLE_CXX"]
    for c in ("/usr/bin/x86_64-linux-gnu-g++-13", "/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return c
    return "g++"


CXX = _cxx()


def cases() -> list[str]:
    return sorted(d for d in os.listdir(CASES)
                  if os.path.isfile(os.path.join(CASES, d, "Chemistry.H")))


def lib_path(case: str) -> str:
    return os.path.join(LIBDIR, f"liboracle_{case}.so")


if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _case_dir(case: str) -> str:
    from vidyut_b200 import build as vbuild
    return vbuild.case_dir(case)


def _case_flags(case: str):
    from vidyut_b200 import build as vbuild
    return vbuild.case_flags(case)


def _stale(case: str) -> bool:
    out = lib_path(case)
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = [os.path.join(HERE, "vd_oracle.cpp"), os.path.join(HERE, "oracle_defaults.H"),
            os.path.join(ROOT, "include", "vidyut_b200.h")]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".H")]
    cdir = _case_dir(case)
    deps += [os.path.join(cdir, f) for f in os.listdir(cdir)]
    return any(os.path.getmtime(p) > t for p in deps)


def build_case(case: str, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = lib_path(case)
    if not force and not _stale(case):
        return out
    inc, srcs = _case_flags(case)
    cmd = [CXX, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           *inc, "-I", HERE, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           os.path.join(HERE, "vd_oracle.cpp"), *srcs, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for oracle case {case}:\n{r.stderr[-6000:]}")
    os.replace(out + ".tmp", out)
    return out


def build_all(force: bool = False) -> list[str]:
    return [build_case(c, force) for c in cases()]


if __name__ == "__main__":
    force = "--force" in sys.argv
    only = [a for a in sys.argv[1:] if not a.startswith("-")]
    for c in (only or cases()):
        print(build_case(c, force))
