"""Failure paths of the C ABI, made on the host (no GPU fault is caused).

* Out of memory: VD_FAULT_ALLOC_AFTER=n makes the context's allocation after
  the n-th fail exactly as cudaMalloc does on a full device.  vd_create must
  return VD_ERR_OOM with a message, release everything it had made (a
  second context on the same device then builds and steps), and a context
  made afterwards without the variable is unaffected.
* Non-finite state: NaN and inf written into the state through
  vd_set_state are counted by vd_check_state, which returns
  VD_ERR_NONFINITE; the potential solve of a state with a NaN charge is
  reported as not converged (VD_ERR_NOT_CONVERGED), not as a zero residual.
"""
import ctypes

import numpy as np
import pytest

import vidyut_b200 as vb
from vidyut_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small():
    cfg = W.townsend_config(3, 32)
    cfg["n_cell"] = [32, 32, 32]
    return cfg


@pytest.mark.parametrize("after", [0, 3, 12])
def test_injected_out_of_memory_at_create(require_gpu, monkeypatch, after):
    monkeypatch.setenv("VD_FAULT_ALLOC_AFTER", str(after))
    with pytest.raises(vb.VidyutError) as e:
        vb.Vidyut(small())
    assert vb.STATUS[e.value.status] == "VD_ERR_OOM"
    assert "out of memory" in str(e.value)
    monkeypatch.delenv("VD_FAULT_ALLOC_AFTER")
    cfg = small()
    g = vb.Vidyut(cfg)
    g.set_state(0, W.initial_state(cfg, 3))
    st = g.step(1)
    assert st.steps == 1 and st.not_converged == 0
    assert g.check_state() == 0
    g.close()


def test_nonfinite_state_is_counted(require_gpu):
    cfg = small()
    g = vb.Vidyut(cfg)
    S = W.initial_state(cfg, 4)
    g.set_state(0, S)
    assert g.check_state() == 0
    S[0, 5, 6, 7] = np.nan
    S[1, 0, 0, 0] = np.inf
    g.set_state(0, S)
    n = ctypes.c_longlong()
    assert vb.STATUS[g.lib.vd_check_state(g.ctx, ctypes.byref(n))] == "VD_ERR_NONFINITE"
    assert n.value == 2
    g.close()


def test_nan_charge_potential_solve_is_not_converged(require_gpu):
    cfg = small()
    cfg["linsolve_maxiter"] = 5
    g = vb.Vidyut(cfg)
    S = W.initial_state(cfg, 5)
    S[1, 10, 11, 12] = np.nan
    g.set_state(0, S)
    st = g.solve_potential(0.0, allow_unconverged=True)
    assert not st.converged
    with pytest.raises(vb.VidyutError) as e:
        g.solve_potential(0.0)
    assert vb.STATUS[e.value.status] == "VD_ERR_NOT_CONVERGED"
    g.close()
