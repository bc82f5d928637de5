"""The C++ host driver (vidyut_b200/host/vd_run.cpp), which drives a case
library through the C ABI alone, as the reference's executable drives
Vidyut::Evolve from an inputs file (Source/main.cpp).

* CPU: the driver builds against include/vidyut_b200.h and the case
  library, parses a reference-style inputs file with command-line overrides
  and resolves the same configuration as the Python ctypes mirror.
* GPU: three steps run by the driver from the inputs file (initial data from
  the case's amrex_probinit/initdomaindata through vd_init_domain) equal the
  same three steps run through the Python mirror.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import vidyut_b200 as vb
from vidyut_b200 import build

INPUTS = """
# two-species Townsend discharge, 3-D, 24^3 (reference inputs-file syntax)
max_step = 3
stop_time = 1.0
amr.n_cell = 24 24 24
geometry.prob_hi = 0.02 0.02 0.02
vidyut.dt = 5e-13        # fixed step
vidyut.hyp_order = 5
vidyut.weno_scheme = 3
vidyut.using_LFA = 1
vidyut.bound_specden = 1
vidyut.gas_temperature = 300.0
vidyut.gas_pressure = 101442.6
vidyut.bg_species_ids = 2
vidyut.pot_bc_lo = 2 2 1
vidyut.pot_bc_hi = 2 2 1
vidyut.voltage_amp_hi = 0.0 0.0 20000.0
prob.nblobs = 2
prob.cx = 0.008 0.012
prob.cy = 0.01 0.011
prob.cz = 0.009 0.012
prob.ampl = 1e18 3e17
prob.sigma = 1e-3 6e-4
"""


def run_host(tmp_path, *extra):
    exe = build.build_host("townsend")
    inp = tmp_path / "inputs"
    inp.write_text(INPUTS)
    return subprocess.run([exe, str(inp), *extra], capture_output=True, text=True, timeout=600)


def test_host_resolves_inputs(tmp_path):
    r = run_host(tmp_path, "vidyut.hyp_order=2", "--check")
    assert r.returncode == 0, r.stderr
    m = re.search(r"dim (\d), n_cell (\d+) (\d+) (\d+), dt ([\de.+-]+), hyp_order (\d), "
                  r"weno_scheme (\d), correctors (\d), max_step (\d+)", r.stdout)
    assert m, r.stdout
    cfg = vb.Config.from_inputs("townsend", INPUTS + "vidyut.hyp_order = 2\n")
    assert int(m.group(1)) == cfg["dim"] == 3
    assert [int(m.group(i)) for i in (2, 3, 4)] == list(cfg["n_cell"])
    assert float(m.group(5)) == cfg["dt"]
    assert int(m.group(6)) == cfg["hyp_order"] == 2   # the command line overrides the file
    assert int(m.group(7)) == cfg["weno_scheme"] and int(m.group(9)) == 3
    assert "case townsend" in r.stdout


def read_dump(path):
    with open(path, "rb") as f:
        assert f.read(4) == b"VDST"
        dim, nx, ny, nz, nc, step = np.frombuffer(f.read(24), dtype=np.int32)
        t = np.frombuffer(f.read(8), dtype=np.float64)[0]
        S = np.frombuffer(f.read(), dtype=np.float64).reshape(nc, nz, ny, nx)
    return S, int(step), float(t)


@pytest.mark.gpu
def test_host_steps_equal_python_mirror(require_gpu, tmp_path):
    out = tmp_path / "final.bin"
    r = run_host(tmp_path, "--dump", str(out))
    assert r.returncode == 0, r.stderr + r.stdout
    assert r.stdout.count("\nstep ") + r.stdout.startswith("step ") == 3, r.stdout
    S, step, t = read_dump(out)
    assert step == 3 and abs(t - 1.5e-12) < 1e-24
    cfg = vb.Config.from_inputs("townsend", INPUTS)
    prob = "\n".join(ln for ln in INPUTS.splitlines() if ln.startswith("prob."))
    g = vb.Vidyut(cfg)
    g.init_domain(prob)
    g.step(3)
    ref = g.get_state()
    g.close()
    assert np.isfinite(S).all()
    for c in range(ref.shape[0]):
        scale = np.max(np.abs(ref[c])) or 1.0
        assert np.max(np.abs(S[c] - ref[c])) <= 1e-13 * scale, c
