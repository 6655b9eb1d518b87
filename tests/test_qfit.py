"""The constant-Q calibration (seiscl_b200.qfit.ConstantQFit) against
SeisCL's own QTAU fit (SeisCL/Q_tau.py:25-127): the values it produced
(tests/golden/qtau.json, written by tests/golden/make_qtau.py) and, where
the reference tree is present, the module itself run live.  The headline
3D benchmark takes its FL and tau from this fit (Q = 50 over 5-40 Hz)."""
import json
import os

import numpy as np
import pytest

from tests.golden.make_qtau import CASES, initial_fl, load_qtau, reference_values

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SEISCL_REFERENCE", "/root/reference")


def ours():
    from seiscl_b200.qfit import ConstantQFit

    out = []
    for qmin, qmax, fmin, fmax, fl0, qs in CASES:
        fit = ConstantQFit(qmin, qmax, fmin, fmax, initial_fl(fl0, fmin, fmax))
        before = [fit.q_to_tau(v) for v in qs]
        fit.optimize()
        out.append(dict(fl=fit.fl(), tau=[fit.q_to_tau(v) for v in qs], tau_before=before))
    return out


def _compare(got, want):
    for g, w in zip(got, want):
        assert np.allclose(g["tau_before"], w["tau_before"], rtol=1e-12, atol=0)
        assert np.allclose(g["fl"], w["fl"], rtol=1e-6, atol=0)
        assert np.allclose(g["tau"], w["tau"], rtol=1e-6, atol=0)


def test_constant_q_fit_matches_golden_values():
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "qtau.json")))
    _compare(ours(), want)


def test_constant_q_fit_matches_reference_module():
    if not os.path.exists(os.path.join(REF, "SeisCL", "Q_tau.py")):
        pytest.skip("reference tree not present")
    _compare(ours(), reference_values(load_qtau(REF)))


def test_benchmark_calibration():
    from seiscl_b200.qfit import constant_q_band

    fl, tau = constant_q_band(2, 50.0, 5.0, 40.0)
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "qtau.json")))[0]
    assert np.allclose(fl, want["fl"], rtol=1e-6)
    assert abs(tau - want["tau"][1]) < 1e-6 * tau
