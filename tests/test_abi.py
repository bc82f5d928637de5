"""C-ABI checks that need no GPU: every function declared in
include/vidyut_b200.h is exported by every case library, the config
interface follows the reference's parameter names and defaults, and the
case tables match the case headers."""
import ctypes
import os
import re

import pytest

import vidyut_b200 as vb
from vidyut_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "vidyut_b200.h")).read()
    return sorted(set(re.findall(r"^vd_status\s+(vd_\w+)\s*\(", hdr, re.M)))


def test_header_declares_the_python_binding_surface():
    assert set(declared_symbols()) == set(vb.EXPORTS)


@pytest.mark.parametrize("case", build.cases())
def test_library_loads_and_exports_every_declared_symbol(case):
    lib = vb.load(case)
    for name in declared_symbols():
        assert hasattr(lib, name), name
    raw = ctypes.CDLL(vb.lib_path(case))
    for name in declared_symbols():
        assert getattr(raw, name) is not None


def test_config_defaults_are_the_references():
    cfg = vb.Config("townsend")
    # Source/Vidyut.H:255-288
    assert cfg["dt"] == 1e-12
    assert cfg["linsolve_reltol"] == 1e-10 and cfg["linsolve_abstol"] == 1e-10
    assert cfg["linsolve_maxiter"] == 100
    assert cfg["linsolve_num_pre_smooth"] == 2 and cfg["linsolve_num_post_smooth"] == 2
    assert cfg["hyp_order"] == 1 and cfg["weno_scheme"] == 3
    assert cfg["min_electron_density"] == 1e12 and cfg["min_species_density"] == 1e-20
    assert cfg["num_timestep_correctors"] == 1


def test_config_set_by_inputs_names():
    cfg = vb.Config.from_inputs("townsend", """
amr.n_cell = 64 32 16
vidyut.hyp_order = 5
vidyut.pot_bc_lo = 2 2 1   # comment
vidyut.voltage_amp_hi = 0 0 2e4
vidyut.bg_species_ids = 2
unknown.key = 3
""")
    assert cfg["n_cell"] == [64, 32, 16]
    assert cfg["hyp_order"] == 5
    assert cfg["pot_bc_lo"] == [2, 2, 1]
    assert cfg["voltage_amp_hi"][2] == 2e4
    assert cfg["num_bg_species"] == 1 and cfg["bg_species_ids"][0] == 2
    with pytest.raises(vb.VidyutError):
        cfg.set("vidyut.no_such_key", "1")


def test_case_tables():
    info = vb.case_info("townsend")
    assert info["num_species"] == 3 and info["names"] == ["E", "ION", "N"]
    assert info["charge"] == [-1, 1, 0]
    # Source/VarDefines.H:5-38 numbering
    assert info["een_id"] == 3 and info["etemp_id"] == 4 and info["pot_id"] == 5
    assert info["efx_id"] == 6 and info["ref_id"] == 12 and info["nvar"] == 25


def test_create_rejects_bad_parameters_without_gpu_work():
    cfg = vb.Config("townsend")
    cfg["hyp_order"] = 3  # Source/Vidyut.cpp:458-461 aborts on this
    with pytest.raises(vb.VidyutError) as e:
        vb.Vidyut(cfg)
    assert e.value.status == 1
