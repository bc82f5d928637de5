"""A case directory written in the reference's conventions, built unchanged.

`tests/amrex_style/mms1/` is MMS1 written the way the reference writes a case
directory: AMReX headers and types (`amrex::Real`, `Array4<Real>`,
`GpuArray<Real, AMREX_SPACEDIM>`, `AMREX_D_DECL`), species names in a
`Chemistry.cpp`, `amrex_probinit(ProbParm&, ProbParm&)` over
`amrex::ParmParse` with `Gpu::htod_memcpy`, `initdomaindata` over
`lbound`/`ubound`, and boundary hooks with the three integrated-current
arguments.  It travels with the repository (unlike the reference's own
directories, `tests/test_reference_cases.py`), so the compatibility headers
(`vidyut_b200/compat/`) are exercised on the GPU too:

* CPU: it builds for sm_100a and for the oracle, reports its species from
  `Chemistry.cpp`, and the oracle's states equal the restated
  `vidyut_b200/cases/mms1` bit for bit over 100 steps;
* GPU: the library's states equal the library's run of the restated case
  bit for bit, and the oracle's within 1e-9 per field after 100 steps (the
  bound of the restated case's own parity test, tests/test_parity_gpu.py:
  both solvers stop at their tolerance every step).
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import vidyut_b200 as vb
from oracle import build as obuild
from oracle.oracle import Oracle
from tests.cases import mms1_config
from vidyut_b200 import build
from vidyut_b200.compare import field_error

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = "amx_mms1"


@pytest.fixture(scope="module")
def built():
    build.register_case(CASE, os.path.join(HERE, "amrex_style", "mms1"))
    with ThreadPoolExecutor(2) as ex:
        list(ex.map(lambda f: f(CASE), (build.build_case, obuild.build_case)))
    return CASE


def config(case, n=32, hyp=5):
    ref = mms1_config(n, hyp)
    cfg = vb.Config(case)
    for name, _ in vb.vd_config._fields_:
        setattr(cfg.c, name, getattr(ref.c, name))
    return cfg


def run(runner, steps):
    runner.init_domain("prob.axial_dir = 0")
    runner.step(steps)
    S = runner.get_state()
    runner.close()
    return S


def test_amrex_style_case_builds_and_equals_restatement_on_oracle(built):
    info = vb.case_info(built)
    assert info["names"] == ["E", "NI"] and info["charge"] == [-1, -1]
    S = run(Oracle(config(built)), 100)
    T = run(Oracle(mms1_config(32, 5)), 100)
    assert np.array_equal(S, T)


@pytest.mark.gpu
def test_amrex_style_case_on_gpu(require_gpu, built):
    G = run(vb.Vidyut(config(built)), 100)
    O = run(Oracle(config(built)), 100)
    R = run(vb.Vidyut(mms1_config(32, 5)), 100)
    assert np.array_equal(G, R)
    info = vb.case_info(built)
    for c in (1, info["pot_id"]):
        assert field_error(O[c], G[c])[1] < 1e-9, c
