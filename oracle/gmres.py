"""Oracle: restarted GMRES(40), the linear solver that replaces cuDSS in this package.

Test infrastructure only (see ``oracle/__init__``).  The reference factorises
A = I + alpha*J with cuDSS LU (reference bdf.cu:150-180); ``rdcu_b200/csrc/bdf.cu``
solves A x = b with restarted GMRES(40) instead, because cuDSS is not installed.  This
module restates that solver without a preconditioner, which is the library's form for
more than four fields.  It lets the oracle BDF run with the same inexact solves, so a
CPU test can check that they leave the stepper's decisions those of the direct solve.

The recurrence is the library's:
* the residual target is 1e-12 * ||b||, and the first guess is x = 0;
* each Arnoldi step makes two classical Gram-Schmidt passes, and the Hessenberg column
  is the sum of the two passes' coefficients;
* Givens rotations update the least-squares residual g;
* a cycle stops when |g[j+1]| <= tol, when ||w|| = 0, after 40 columns, or after 400
  iterations in total;
* back-substitution gives y, and x += V y;
* a restart recomputes r = b - A x, and there are at most 50 cycles.
"""
from __future__ import annotations

import math

import numpy as np

RESTART = 40
LIN_TOL = 1e-12
MAX_ITERS = 400
MAX_CYCLES = 50


class Gmres:
    """x = A^-1 b by restarted GMRES(40); ``stats`` counts iterations, solves, cycles."""

    def __init__(self, A, stats: dict | None = None):
        self.A = A
        self.stats = stats if stats is not None else {"iterations": 0, "solves": 0, "cycles": 0}

    def solve(self, b: np.ndarray) -> np.ndarray:
        A, m = self.A, RESTART
        x = np.zeros(b.size)
        self.stats["solves"] += 1
        beta0 = math.sqrt(float(b @ b))
        if not beta0 > 0:
            return x
        tol = LIN_TOL * beta0
        r, beta, total = b, beta0, 0
        for cycle in range(MAX_CYCLES):
            if total >= MAX_ITERS:
                break
            if cycle > 0:
                r = b - A @ x
                beta = math.sqrt(float(r @ r))
                if not beta > tol:
                    break
            self.stats["cycles"] += 1
            V = [r / beta]
            H = np.zeros((m, m))
            cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
            g[0] = beta
            jdone, conv = 0, False
            for j in range(m):
                w = A @ V[j]
                h = np.zeros(j + 1)
                for _ in range(2):
                    d = np.array([float(V[k] @ w) for k in range(j + 1)])
                    h = h + d
                    for k in range(j + 1):
                        w = w - d[k] * V[k]
                hn = math.sqrt(float(w @ w))
                total += 1
                col = list(h)
                for k in range(j):
                    a = cs[k] * col[k] + sn[k] * col[k + 1]
                    col[k + 1] = -sn[k] * col[k] + cs[k] * col[k + 1]
                    col[k] = a
                den = math.sqrt(col[j] * col[j] + hn * hn)
                cs[j] = col[j] / den if den > 0 else 1.0
                sn[j] = hn / den if den > 0 else 0.0
                col[j] = den
                g[j + 1] = -sn[j] * g[j]
                g[j] = cs[j] * g[j]
                H[:j + 1, j] = col
                jdone = j + 1
                met = abs(g[j + 1]) <= tol or not hn > 0
                if met or total >= MAX_ITERS:
                    conv = met
                    break
                V.append(w * (1.0 / hn))  # the library scales by the reciprocal (bdf.cu k_gm_update)
            y = np.zeros(jdone)
            for k in range(jdone - 1, -1, -1):
                acc = g[k]
                for q in range(k + 1, jdone):
                    acc -= H[k, q] * y[q]
                y[k] = acc / H[k, k] if H[k, k] != 0 else 0.0
            for k in range(jdone):
                x = x + y[k] * V[k]
            if conv:
                break
        self.stats["iterations"] += total
        return x
