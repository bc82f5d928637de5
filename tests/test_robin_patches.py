"""Potential walls of Dirichlet patches in a Neumann face (Robin sides).

The electrode layout of the solver workload's user potential callback
(vidyut_b200/cases/mgsolve/UserFunctions.H, the geometry of the reference's
test/models/Ar_RF_Sputter3d potential callback on the unit cube): two disc
electrodes at +-60 V in the low-z wall and a grounded disc substrate in the
high-z wall, (a, b, f) = (1, 0, V) on the discs and (0, 1, 0) elsewhere on
those walls, Neumann on x and y.

The multigrid hierarchy coarsens such a side by the fine faces' boundary
conductance (a coarse face half covered by an electrode is Dirichlet); the
earlier mean of a and b turned the coarse walls nearly Neumann and the
V-cycle diverged.  A residual that went non-finite reads as not converged.

CPU: the oracle converges within a bound of V-cycles; with no space charge
the potential obeys the maximum principle and the layout's antisymmetry
phi(x, y, z) = -phi(x, 1 - y, z); a NaN in the charge is reported as not
converged.  GPU: the library against the oracle (FP64 and FP32-refined) with
the workload's seeded charge, and a NaN reported as not converged."""
import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

ROBIN_Z = dict(user_defined_potential=1, pot_bc_lo=[2, 2, 4], pot_bc_hi=[2, 2, 4])


def electrodes(n, **kw):
    return W.mgsolve_config(n, **{**ROBIN_Z, **kw})


def neutral_state(cfg):
    S = W.mgsolve_state(cfg, 1)
    S[1] = S[0]
    return S


def solve(runner, cfg, S, **kw):
    runner.init_domain("")
    runner.set_state(0, S)
    st = runner.solve_potential(0.0, **kw)
    return st, runner.get_state(runner.info["pot_id"], 1)


def test_oracle_electrode_walls_converge():
    for n in (32, 64):
        cfg = electrodes(n, linsolve_reltol=1e-10, linsolve_abstol=0.0)
        o = Oracle(cfg)
        st, _ = solve(o, cfg, W.mgsolve_state(cfg, 1))
        o.close()
        assert st.converged and st.iterations <= 25, (n, st.iterations)


def test_oracle_electrode_potential_symmetry():
    cfg = electrodes(32, linsolve_reltol=1e-12, linsolve_abstol=0.0)
    o = Oracle(cfg)
    st, phi = solve(o, cfg, neutral_state(cfg))
    o.close()
    assert st.converged
    phi = phi.reshape(32, 32, 32)            # (z, y, x)
    assert phi.max() < 60.0 and phi.min() > -60.0
    assert phi.max() > 30.0                  # the electrodes drive it
    assert np.abs(phi + phi[:, ::-1, :]).max() < 1e-9 * 60.0


def test_oracle_nan_charge_is_not_converged():
    cfg = electrodes(16)
    S = W.mgsolve_state(cfg, 1)
    S[1, 5, 7, 3] = np.nan
    o = Oracle(cfg)
    st, _ = solve(o, cfg, S)
    o.close()
    assert not st.converged


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [vb.VD_MG_FP64, vb.VD_MG_FP32_REFINED])
def test_gpu_electrode_walls_against_oracle(require_gpu, precision):
    cfg_o = electrodes(64, linsolve_reltol=1e-12, linsolve_abstol=0.0)
    S = W.mgsolve_state(cfg_o, 1)
    o = Oracle(cfg_o)
    so, phi_o = solve(o, cfg_o, S)
    o.close()
    cfg_g = electrodes(64, linsolve_reltol=1e-12, linsolve_abstol=0.0, mg_precision=precision)
    g = vb.Vidyut(cfg_g)
    sg, phi_g = solve(g, cfg_g, S)
    g.close()
    assert so.converged and sg.converged
    if precision == vb.VD_MG_FP64:
        assert abs(sg.iterations - so.iterations) <= 1, (sg.iterations, so.iterations)
    assert field_error(phi_o, phi_g)[1] < 1e-10


@pytest.mark.gpu
def test_gpu_nan_charge_is_not_converged(require_gpu):
    cfg = electrodes(32, linsolve_maxiter=8)
    S = W.mgsolve_state(cfg, 1)
    S[1, 5, 7, 3] = np.nan
    g = vb.Vidyut(cfg)
    st, _ = solve(g, cfg, S, allow_unconverged=True)
    assert not st.converged
    with pytest.raises(vb.VidyutError) as e:
        solve(g, cfg, S)
    assert e.value.status == 3               # VD_ERR_NOT_CONVERGED
    g.close()
