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


class ConstantQFit:
    """Least-squares constant-Q calibration of the relaxation frequencies.

    The procedure of SeisCL's QTAU class (SeisCL/Q_tau.py:25-127): for the
    relaxation times ts_l = 1/(2 pi FL_l), the band-averaged 1/Q over
    [fmin, fmax) (0.1 Hz steps) is tabulated at 40 log-spaced strengths tau
    between 1/(2 Qmax) and 2/Qmin; ``q_to_tau`` interpolates that table
    linearly in log-log; ``optimize`` moves the ts_l (L-BFGS-B, bounds
    [1e-6, 0.3]) to make log(1/Q) linear in log(tau) with unit slope and a
    small spread across the band, where the spread term is -- as in the
    reference -- the standard deviation of 1/Q at the last tabulated tau
    divided by each tabulated mean, summed.
    """

    def __init__(self, qmin: float, qmax: float, fmin: float, fmax: float, fl):
        self.qmin, self.qmax, self.fmin, self.fmax = float(qmin), float(qmax), float(fmin), float(fmax)
        self.ts = np.array([1.0 / (2.0 * np.pi * f) for f in fl], dtype=np.float64)
        self._table()

    def _inverse_q(self, tau: float, ts):
        w = 2.0 * np.pi * np.arange(self.fmin, self.fmax, 0.1)
        a = np.zeros_like(w)
        b = np.zeros_like(w)
        for t in ts:
            a = a + w ** 2 * t ** 2 / (1.0 + w ** 2 * t ** 2)
            b = b + w * t / (1.0 + w ** 2 * t ** 2)
        return 1.0 / ((1.0 / tau + a) / b)

    def _calibrate(self, ts):
        logt = np.linspace(np.log(1.0 / self.qmax / 2.0), np.log(1.0 / self.qmin * 2.0), 40)
        qi = np.zeros(len(logt))
        spread = 0.0
        for i, lt in enumerate(logt):
            inv = self._inverse_q(np.exp(lt), ts)
            qi[i] = np.average(inv)
            spread = np.std(inv)
        x, y = logt, np.log(qi)
        xm, ym = x.mean(), y.mean()
        slope = np.sum((x - xm) * (y - ym)) / np.sum((x - xm) ** 2)
        return logt, qi, float(np.sum(spread / qi)), float(slope)

    def _table(self):
        logt, qi, _, _ = self._calibrate(self.ts)
        self._logq, self._logt = np.log(qi), logt

    def optimize(self) -> None:
        from scipy.optimize import minimize

        def loss(ts):
            _, _, spread, slope = self._calibrate(ts)
            return (slope - 1.0) ** 2 + spread

        self.ts = np.asarray(minimize(loss, self.ts, bounds=[(1e-6, 0.3)] * len(self.ts)).x, dtype=np.float64)
        self._table()

    def fl(self):
        return [float(1.0 / t / 2.0 / np.pi) for t in self.ts]

    def q_to_tau(self, q: float) -> float:
        return float(np.exp(np.interp(np.log(1.0 / q), self._logq, self._logt)))


def constant_q_band(L: int, q: float, fmin: float, fmax: float, qmin: float = 10.0, qmax: float = 200.0):
    """(FL, tau) of a constant-Q medium over [fmin, fmax]: the relaxation
    frequencies start geometrically spread over the band and are optimised
    by ``ConstantQFit`` (Q range [qmin, qmax]); tau is its Q2tau(q)."""
    fit = ConstantQFit(qmin, qmax, fmin, fmax, band_frequencies(L, fmin, fmax))
    fit.optimize()
    return fit.fl(), fit.q_to_tau(q)
