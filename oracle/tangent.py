"""Oracle: tangent-linear (forward-mode) derivative of fixed-step DP45.

Test infrastructure only (see ``oracle/__init__``).  The reference has no derivatives;
this module differentiates the oracle's restatement of its pseudospectral RHS
(``spectral.rhs``, reference rdcu.cu:151-184) and of the DP45 stage formulas
(reference dp45.cu:34-69, tableau dp45.cu:6-11) by hand, so that the GPU discrete
adjoint can be checked by the duality <w, dyT> = <grad_y0, dy0> + <grad_C, dC>.
"""
from __future__ import annotations

import numpy as np

from . import dp45 as odp
from . import spectral as osp
from .problem import Problem, pow_c


def rhs(y: np.ndarray, prob: Problem, C=None) -> np.ndarray:
    """The dictionary RHS with coefficients C (None: the problem's own)."""
    Q = osp.spectral_Y(y, prob).real
    n, N = prob.n, prob.N
    f = np.zeros((n, N))
    for ti, term in enumerate(prob.terms):
        c = term.C if C is None else C[ti]
        tv = np.ones(N)
        for (k, eta) in term.pairs:
            tv = tv * pow_c(Q[k], 1.0 * eta)
        f[term.field] += c * tv
    return f.reshape(-1)


def rhs_jvp(y: np.ndarray, dy: np.ndarray, prob: Problem, C=None, dC=None) -> np.ndarray:
    """d/de f(y + e dy; C + e dC) at e = 0.  The derivative blocks are linear in y
    (Re IFFT(M FFT y)), so dQ_k = Q_k(dy); each monomial follows the product rule."""
    Q = osp.spectral_Y(y, prob).real
    dQ = osp.spectral_Y(dy, prob).real
    n, N = prob.n, prob.N
    df = np.zeros((n, N))
    for ti, term in enumerate(prob.terms):
        c = term.C if C is None else C[ti]
        P = np.ones(N)
        dP = np.zeros(N)
        for (k, eta) in term.pairs:
            if eta == 0:
                continue
            qe = pow_c(Q[k], 1.0 * eta)
            dP = dP * qe + P * eta * pow_c(Q[k], eta - 1.0) * dQ[k]
            P = P * qe
        df[term.field] += c * dP
        if dC is not None:
            df[term.field] += dC[ti] * P
    return df.reshape(-1)


_A = [[], odp.A1, odp.A2, odp.A3, odp.A4, odp.A5, odp.B1]


def dp45_tlm(y0, dy0, hs, prob: Problem, C=None, dC=None):
    """Fixed-step DP45 over the step sizes hs with its tangent: returns (yT, dyT)."""
    y = np.array(y0, np.float64)
    dy = np.array(dy0, np.float64)
    for h in hs:
        k, dk = [], []
        for i in range(7):
            if i == 0:
                Yi, dYi = y, dy
            else:
                a = _A[i]
                Yi = y + h * sum(a[j] * k[j] for j in range(i))
                dYi = dy + h * sum(a[j] * dk[j] for j in range(i))
            if i == 6:  # stage 7 state is the new y (b row = a_7j)
                y, dy = Yi, dYi
                break
            k.append(rhs(Yi, prob, C))
            dk.append(rhs_jvp(Yi, dYi, prob, C, dC))
    return y, dy


def dp45_fixed(y0, hs, prob: Problem, C=None):
    """Fixed-step DP45 over the step sizes hs (no tangent)."""
    y = np.array(y0, np.float64)
    for h in hs:
        k = []
        for i in range(7):
            Yi = y if i == 0 else y + h * sum(_A[i][j] * k[j] for j in range(i))
            if i == 6:
                y = Yi
                break
            k.append(rhs(Yi, prob, C))
    return y
