"""Constant-Q calibration of the generalized standard linear solid.

For L relaxation mechanisms with relaxation frequencies FL (tau_sigma_l =
1/(2 pi FL_l)) and a relaxation strength tau, the quality factor at angular
frequency w is

    Q(w) = (1/tau + sum_l w^2 ts_l^2/(1 + w^2 ts_l^2)) / sum_l w ts_l/(1 + w^2 ts_l^2)

(Blanch, Robertsson & Symes 1995; the same relation SeisCL's Q_tau.py uses,
SeisCL/Q_tau.py:53-67).  ``q_to_tau`` returns the tau whose band-averaged 1/Q
over [fmin, fmax] equals 1/Q0, found by bisection.
"""
from __future__ import annotations

import numpy as np


def inverse_q(tau: float, fl, fmin: float, fmax: float, df: float = 0.1) -> float:
    w = 2 * np.pi * np.arange(fmin, fmax, df)
    ts = 1.0 / (2 * np.pi * np.asarray(fl, dtype=np.float64))
    a = np.zeros_like(w)
    b = np.zeros_like(w)
    for t in ts:
        a += w ** 2 * t ** 2 / (1.0 + w ** 2 * t ** 2)
        b += w * t / (1.0 + w ** 2 * t ** 2)
    q = (1.0 / tau + a) / b
    return float(np.mean(1.0 / q))


def q_to_tau(q0: float, fl, fmin: float, fmax: float) -> float:
    lo, hi = 1e-8, 10.0
    target = 1.0 / q0
    for _ in range(200):
        mid = np.sqrt(lo * hi)
        if inverse_q(mid, fl, fmin, fmax) < target:
            lo = mid
        else:
            hi = mid
    return float(np.sqrt(lo * hi))


def band_frequencies(L: int, fmin: float, fmax: float):
    """Relaxation frequencies spread geometrically over the band."""
    r = fmax / fmin
    return [float(fmin * r ** ((2 * k + 1) / (2.0 * L))) for k in range(L)]
