"""Oracle: the Dormand-Prince 4(5) stepper.

Test infrastructure only (see ``oracle/__init__``).  Restates reference ``dp45.cu``:
coefficient tables (dp45.cu:6-21), stage kernels (dp45.cu:34-69), ``interpolate``
(dp45.cu:70-76), ``error`` (dp45.cu:79-84), ``dp45_step`` (dp45.cu:87-147),
``dp45_eval`` (dp45.cu:149-152) and ``dp45_run`` (dp45.cu:154-169).
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np

# dp45.cu:6-13
A1 = [1.0 / 5]
A2 = [3.0 / 40, 9.0 / 40]
A3 = [44.0 / 45, -56.0 / 15, 32.0 / 9]
A4 = [19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729]
A5 = [9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656]
B1 = [35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84]
CC = [0.0, 1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1.0]
E = [-71.0 / 57600, 0, 71.0 / 16695, -71.0 / 1920, 17253.0 / 339200, -22.0 / 525, 1.0 / 40]
# dp45.cu:15-21 (dense-output polynomial coefficients, rows k1..k7, columns x^1..x^4)
P = [
    [1.0, -8048581381.0 / 2820520608, 8663915743.0 / 2820520608, -12715105075.0 / 11282082432],
    [0, 0, 0, 0],
    [0, 131558114200.0 / 32700410799, -68118460800.0 / 10900136933, 87487479700.0 / 32700410799],
    [0, -1754552775.0 / 470086768, 14199869525.0 / 1410260304, -10690763975.0 / 1880347072],
    [0, 127303824393.0 / 49829197408, -318862633887.0 / 49829197408, 701980252875.0 / 199316789632],
    [0, -282668133.0 / 205662961, 2019193451.0 / 616988883, -1453857185.0 / 822651844],
    [0, 40617522.0 / 29380423, -110615467.0 / 29380423, 69997945.0 / 29380423],
]


class DP45:
    """State of the reference stepper (its file-static globals, dp45.cu:24-31)."""

    def __init__(self, y0: np.ndarray, atol: float, rtol: float, fixed: bool,
                 dydt: Callable[[float, np.ndarray], np.ndarray]):
        # dp45_init (dp45.cu:171-225)
        self.y = np.array(y0, np.float64)
        self.N = self.y.size
        self.atl, self.rtl, self.fixed = atol, rtol, bool(fixed)
        self.dydt = dydt
        self.k = [None] * 7
        self.ylast = self.y.copy()
        self.t_last = 0.0
        self.ytemp = None
        self.last_norm = None

    def step(self, t: float, h: float, hmin: float, hmax: float):
        """dp45_step (dp45.cu:87-147).  Returns (accepted, t, h)."""
        y, k = self.y, self.k
        f = self.dydt
        k[1] = f(t + h * CC[1], y + h * A1[0] * k[0])
        k[2] = f(t + h * CC[2], y + h * (A2[0] * k[0] + A2[1] * k[1]))
        k[3] = f(t + h * CC[3], y + h * (A3[0] * k[0] + A3[1] * k[1] + A3[2] * k[2]))
        k[4] = f(t + h * CC[4], y + h * (A4[0] * k[0] + A4[1] * k[1] + A4[2] * k[2]
                                          + A4[3] * k[3]))
        k[5] = f(t + h * CC[5], y + h * (A5[0] * k[0] + A5[1] * k[1] + A5[2] * k[2]
                                          + A5[3] * k[3] + A5[4] * k[4]))
        ytemp = y + h * (B1[0] * k[0] + B1[1] * k[1] + B1[2] * k[2] + B1[3] * k[3]
                         + B1[4] * k[4] + B1[5] * k[5])
        k[6] = f(t + h, ytemp)
        self.ytemp = ytemp
        if self.fixed:
            self.t_last = t
            self.ylast = y
            self.y = ytemp
            return True, t + h, h
        yerr = h * (E[0] * k[0] + E[1] * k[1] + E[2] * k[2] + E[3] * k[3] + E[4] * k[4]
                    + E[5] * k[5] + E[6] * k[6]) / (
            self.atl + self.rtl * np.maximum(np.abs(y), np.abs(ytemp)))
        with np.errstate(all="ignore"):
            norm = float(np.sqrt(np.sum(yerr * yerr)))
            norm /= math.pow(self.N, 0.5)
            self.last_norm = norm
            try:
                factor = 0.9 * math.pow(norm, -0.2)
            except (ZeroDivisionError, ValueError, OverflowError):
                factor = math.inf if norm == 0 else math.nan
        if math.isnan(factor):
            factor = 0.2
        if norm < 1:
            self.t_last = t
            self.ylast = y
            self.y = ytemp
            t = t + h
            if factor > 10:
                factor = 10
            h *= factor
            if h > hmax:
                h = hmax
            return True, t, h
        elif factor < 1:
            if factor < 0.2:
                factor = 0.2
            h *= factor
        return False, t, h

    def eval(self, t: float, t_eval: float) -> np.ndarray:
        """dp45_eval / interpolate (dp45.cu:70-76,149-152), evaluated in the kernel's
        order: y + h*(x*S1 + x^2*S2 + x^3*S3 + x^4*S4)."""
        k = self.k
        h = t - self.t_last
        x = (t_eval - self.t_last) / h
        S = []
        for p in range(4):
            S.append(P[0][p] * k[0] + P[1][p] * k[1] + P[2][p] * k[2] + P[3][p] * k[3]
                     + P[4][p] * k[4] + P[5][p] * k[5] + P[6][p] * k[6])
        return self.ylast + h * (x * S[0] + x * x * S[1] + x * x * x * S[2]
                                 + x * x * x * x * S[3])

    def run(self, t: float, h: float, hmin: float, hmax: float, t1: float, step_eval,
            max_attempts: int | None = None):
        """dp45_run (dp45.cu:154-169): FSAL k1, then attempt until t >= t1 or h <= hmin;
        ``step_eval(t, h, y, success)`` after every attempt; k1 <- k7 on success."""
        self.k[0] = self.dydt(t, self.y)
        attempts = 0
        while t < t1 and h > hmin:
            ok, t, h = self.step(t, h, hmin, hmax)
            step_eval(t, h, self.y, ok)
            if ok:
                self.k[0] = self.k[6]
            attempts += 1
            if max_attempts is not None and attempts >= max_attempts:
                break
        return t, h
