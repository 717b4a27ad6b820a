"""Oracle: the variable-order NDF/BDF stepper (ode15s style) on the FD discretisation.

Test infrastructure only (see ``oracle/__init__``).  Restates reference ``bdf.cu``:
constants (bdf.cu:8-9,23), ``makeRU`` (bdf.cu:35-69), kernels ``updateD``, ``errscale``,
``step0``, ``rhs``, ``interpolate``, ``scale_err`` (bdf.cu:72-132), ``bdf_step``
(bdf.cu:135-323), ``bdf_eval`` (bdf.cu:325-328), ``bdf_run`` (bdf.cu:330-389) and the
tolerance set-up of ``bdf_init`` (bdf.cu:391-401).  The cuDSS LU of A = I + alpha*J is
replaced by scipy's SuperLU on the same CSR matrix (a direct solve, like cuDSS), or,
with ``linear="gmres"``, by the restarted GMRES(40) of ``oracle.gmres`` (the library's
solver in its unpreconditioned form).
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

KAPPA = [0.0, -0.1850, -1.0 / 9, -0.0823, -0.0415, 0.0]
GAMMA = [0.0, 1.0, 1.0 + 1.0 / 2, 1.0 + 1.0 / 2 + 1.0 / 3, 1.0 + 1.0 / 2 + 1.0 / 3 + 1.0 / 4,
         1.0 + 1.0 / 2 + 1.0 / 3 + 1.0 / 4 + 1.0 / 5]
NWIT = 4


def make_RU(order: int, factor: float) -> np.ndarray:
    """makeRU (bdf.cu:35-69): R[i][j] = prod_{k<i} (k - factor*j)/max(k,1) / max(i,1),
    U the same with factor 1, RU = R @ U; returned flat (order+1)^2 row-major."""
    m = order + 1
    R = np.zeros((m, m))
    U = np.zeros((m, m))
    for i in range(m):
        for j in range(m):
            prod = 1.0 / max(i, 1)
            for k in range(i):
                prod *= (k - factor * j) / max(k, 1)
            R[i, j] = prod
    for i in range(m):
        for j in range(m):
            prod = 1.0 / max(i, 1)
            for k in range(i):
                prod *= (k - j) * 1.0 / max(k, 1)
            U[i, j] = prod
    RU = np.zeros((m, m))
    for i in range(m):
        for j in range(m):
            acc = 0.0
            for k in range(m):
                acc += R[i, k] * U[k, j]
            RU[i, j] = acc
    return RU


def ntol_for(rtol: float) -> float:
    """bdf_init (bdf.cu:395-401)."""
    ntol = 0.03
    if math.pow(rtol, 0.5) < 0.03:
        ntol = math.pow(rtol, 0.5)
    if 10 * math.pow(2, -52) / rtol > ntol:
        ntol = 10 * math.pow(2, -52) / (rtol + math.pow(2, -52))
    return ntol


def _nrm2(x: np.ndarray) -> float:
    return float(np.sqrt(np.sum(x * x)))


class BDF:
    """State of the reference stepper (its file-static globals, bdf.cu:11-32)."""

    def __init__(self, D0: np.ndarray, order: int, atol: float, rtol: float, fixed: bool,
                 dydt: Callable[[float, np.ndarray], np.ndarray],
                 jac: Callable[[float, np.ndarray], tuple], linear: str = "lu"):
        # D has 8 slots (bdf.cu:416); slots 0..order come from the caller (bdf.cu:449)
        self.N = D0[0].size
        self.D = [np.zeros(self.N) for _ in range(8)]
        for i in range(order + 1):
            self.D[i] = np.array(D0[i], np.float64)
        self.order = order
        self.atl, self.rtl, self.fixed = atol, rtol, bool(fixed)
        self.dydt, self.jacf = dydt, jac
        self.ntol = ntol_for(rtol)
        self.refactor, self.rejac = 1, 1
        self.nconststeps = 0.0
        self.J = None
        self.lu = None
        if linear not in ("lu", "gmres"):
            raise ValueError("linear solver: 'lu' or 'gmres'")
        self.linear = linear
        self.lin_stats = {"iterations": 0, "solves": 0, "cycles": 0}

    def _set_jac(self, t, y):
        rows, cols, vals = self.jacf(t, y)
        self.J = sp.csr_matrix((vals, cols, rows), shape=(self.N, self.N))

    def _refactor(self, alpha):
        A = sp.identity(self.N, format="csr") + alpha * self.J
        if self.linear == "gmres":
            from oracle.gmres import Gmres

            self.lu = Gmres(A, self.lin_stats)
        else:
            self.lu = spla.splu(A.tocsc())

    def _update_D(self, factor):
        RU = make_RU(self.order, factor)
        m = self.order + 1
        Dnew = []
        for k in range(m):
            val = np.zeros(self.N)
            for j in range(m):
                val = val + RU[j, k] * self.D[j]
            Dnew.append(val)
        for k in range(m):
            self.D[k] = Dnew[k]

    def setup(self, t: float, h: float):
        """bdf_run set-up (bdf.cu:333-374): f and J at D_0; order 0 -> D_1 = h f, order 1."""
        f = self.dydt(t, self.D[0])
        self._set_jac(t, self.D[0])
        if self.order == 0:
            self.D[1] = f * h
            self.order = 1

    def step(self, t: float, h: float, hmin: float, hmax: float):
        """bdf_step (bdf.cu:135-323).  Returns (accepted, t, h)."""
        N, D, order = self.N, self.D, self.order
        converged = False
        it = 0
        dnorm = dnormold = rate = 0.0
        factor = 1.0
        h0 = h
        ytemp = D[0].copy()
        for j in range(1, order + 1):
            ytemp = ytemp + D[j]
        yscale = self.atl + self.rtl * np.abs(ytemp)
        d = np.zeros(N)
        sqN = math.pow(N, 0.5)
        for it in range(NWIT):
            f = self.dydt(t + h, ytemp)
            if self.refactor:
                alpha = -h / ((1 - KAPPA[order]) * GAMMA[order])
                self._refactor(alpha)
                self.refactor = 0
            al = (1 - KAPPA[order]) * GAMMA[order]
            b = h / al * f
            for j in range(1, order + 1):
                b = b - D[j] * GAMMA[j] / al
            b = b - d
            dd = self.lu.solve(b)
            yerr = dd / yscale
            dnorm = _nrm2(yerr) / sqN
            if dnormold > 0:
                rate = dnorm / dnormold
            if rate >= 1:
                break
            if math.pow(rate, NWIT - it) / (1 - rate) * dnorm > self.ntol:
                break
            if dnormold > 0 and rate / (1 - rate) * dnorm < self.ntol:
                converged = True
                break
            ytemp = ytemp + dd
            d = d + dd
            dnormold = dnorm
        else:
            it = NWIT

        if not converged:
            if self.rejac:
                yp = D[0].copy()
                for j in range(1, order + 1):
                    yp = yp + D[j]
                self._set_jac(t + h, yp)
                self.refactor = 1
                self.rejac = 0
                return False, t, h
            elif not self.fixed:
                factor = 0.5
                h *= factor
                if h < hmin:
                    return False, t, h
                self._update_D(factor)
                self.refactor = 1
                self.nconststeps = 0.0
                return False, t, h

        if self.fixed:
            D[0] = ytemp.copy()
            h = h0
            return True, t + h, h

        safety = (2 * NWIT + 1) * 0.9 / (2 * NWIT + it + 1)
        yscale = self.atl + self.rtl * np.abs(ytemp)
        errnorm = _nrm2(d / yscale)
        errnorm *= (KAPPA[order] * GAMMA[order] + 1.0 / (order + 1)) / sqN
        with np.errstate(all="ignore"):
            factor = safety * _pow(errnorm, -1.0 / (order + 1))
        if errnorm > 1:
            if factor < 0.2:
                factor = 0.2
            h = h * factor
            if h < hmin:
                return False, t, h
            self._update_D(factor)
            self.refactor = 1
            self.nconststeps = 0.0
            return False, t, h

        t = t + h
        D[0] = ytemp.copy()
        self.rejac = 1
        D[order + 2] = d - D[order + 1]
        D[order + 1] = d.copy()
        for i in range(order, 0, -1):
            D[i] = D[i] + D[i + 1]
        self.nconststeps += 1
        if self.nconststeps > order:
            errm, errp, fm, fp = math.inf, math.inf, 0.0, 0.0
            if order > 1:
                errm = _nrm2(D[order] / yscale)
                errm *= (KAPPA[order - 1] * GAMMA[order - 1] + 1.0 / order) / sqN
                fm = safety * _pow(errm, -1.0 / order)
            if order < 5:
                errp = _nrm2(D[order + 2] / yscale)
                errp *= (KAPPA[order + 1] * GAMMA[order + 1] + 1.0 / (order + 2)) / sqN
                fp = safety * _pow(errp, -1.0 / (order + 2))
            dorder = 0
            if order > 1 and fm > factor and fm > fp:
                factor = fm
                dorder = -1
            elif order < 5 and fp > factor:
                factor = fp
                dorder = 1
            if factor > 10:
                factor = 10
            if h * factor > hmax:
                factor = hmax / h
                h = hmax
            else:
                h = h * factor
            self.order = order + dorder
            self._update_D(factor)
            self.nconststeps = 0.0
            self.refactor = 1
        return True, t, h

    def eval(self, t: float, h: float, t_eval: float) -> np.ndarray:
        """bdf_eval / interpolate (bdf.cu:115-125,325-328)."""
        y = self.D[0].copy()
        factor = 1.0
        for j in range(1, self.order + 1):
            factor *= (t_eval - t + j * h) / (j * h)
            y = y + self.D[j] * factor
        return y

    def run(self, t, h, hmin, hmax, t1, step_eval, max_attempts=None):
        """bdf_run loop (bdf.cu:376-383)."""
        self.setup(t, h)
        attempts = 0
        while t < t1 and h > hmin:
            ok, t, h = self.step(t, h, hmin, hmax)
            step_eval(t, h, self.D[0], ok)
            attempts += 1
            if max_attempts is not None and attempts >= max_attempts:
                break
        return t, h


def _pow(x: float, e: float) -> float:
    try:
        return math.pow(x, e)
    except (ZeroDivisionError, ValueError, OverflowError):
        if x == 0:
            return math.inf
        return math.nan
