"""Pins the CPU oracle to the reference's own known-answer tests.

The reference ships no numeric golden outputs for this path; its
verification cases state analytic solutions:
  * MMS1 (test/verification/MMS1/README.md): steady n = x^2,
    phi = (x^4 - x)/12; the reference's CI bound for the MMS family is a
    relative error of 1e-3 (test/verification/MMS2/l2err/l2err.cpp:176-194);
  * Advect (test/verification/Advect/get_error_1d.py): the WENO5 solution
    of sin(pi x - sin(pi x)/pi) advected at unit speed, whose convergence
    order the case exists to show.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.cases import (ADVECT_PROB, advect_config, advect_error, mms1_config,
                         mms1_errors)


def run_mms1(n, hyp):
    o = Oracle(mms1_config(n, hyp))
    o.init_domain("prob.axial_dir = 0")
    o.step(100)
    return mms1_errors(o.get_state(), n)


@pytest.mark.parametrize("hyp", [1, 2, 5])
def test_mms1_steady_state_within_reference_bound(hyp):
    en, ep = run_mms1(32, hyp)
    assert en < 1e-3 * 2 and ep < 1e-3, (en, ep)


def test_mms1_weno5_second_order_convergence():
    e16 = run_mms1(16, 5)
    e32 = run_mms1(32, 5)
    e64 = run_mms1(64, 5)
    for a, b in ((e16, e32), (e32, e64)):
        assert np.log2(a[0] / b[0]) > 1.8
        assert np.log2(a[1] / b[1]) > 1.8


def run_advect(n, weno, T=0.5, dt=2.5e-4):
    o = Oracle(advect_config(n, dt, weno))
    o.init_domain(ADVECT_PROB)
    o.step(int(round(T / dt)))
    return advect_error(o.get_state(), n, T)


@pytest.mark.parametrize("weno,order", [(1, 3.9), (2, 4.7), (3, 4.8)])
def test_advect_weno_convergence_order(weno, order):
    e = [run_advect(n, weno) for n in (20, 40, 80)]
    assert e[2] < 1e-5
    assert np.log2(e[1] / e[2]) > order, e
