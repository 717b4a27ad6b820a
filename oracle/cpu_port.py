"""CPU port of the hot path, used as the timed host baseline of bench.py -- TEST/BENCH
INFRASTRUCTURE ONLY (see oracle/__init__).

The same pseudospectral dictionary RHS as oracle.spectral (reference rdcu.cu:78-184),
restated for speed on the host: real-to-complex FFTs with scipy.fft on all cores
(FFTW is not installed; scipy's pocketfft stands in), the reference's multipliers in
their Hermitian form (Re(IFFT(M U)) = IFFT((M(k)+conj(M(-k)))/2 U)), linear single-
derivative terms summed in spectral space, and the DP45 controller of oracle.dp45.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np
import scipy.fft as sfft

from . import dp45 as odp
from .problem import PI, Problem, cgle_terms
from .spectral import freqs


def _herm_multiplier(prob: Problem, yind: int) -> np.ndarray:
    """Real-part multiplier of Y block yind on the rfftn half spectrum (last axis halved)."""
    ndim = prob.ndim
    shape = list(prob.Ns)
    shape[-1] = prob.Ns[-1] // 2 + 1

    def kax(a, neg):
        N = prob.Ns[a]
        k = freqs(N, prob.Ls[a])
        idx = np.arange(N) if a < ndim - 1 else np.arange(shape[-1])
        if neg:
            idx = (N - idx) % N
        sh = [1] * ndim
        sh[a] = len(idx)
        return k[idx].reshape(sh)

    if yind == 0:
        return np.ones(shape)
    if yind <= ndim:
        a = yind - 1
        # i k(n), Hermitian part: i (k(n) - k(-n))/2
        return 1j * 0.5 * (kax(a, False) - kax(a, True)) * np.ones(shape)
    q = yind - ndim - 1
    a, b = q // ndim, q % ndim
    return -0.5 * (kax(a, False) * kax(b, False) + kax(a, True) * kax(b, True)) * np.ones(shape)


class PortRHS:
    def __init__(self, prob: Problem, workers: int):
        self.prob, self.workers = prob, workers
        n = prob.n
        self.fold = [None] * n
        self.needed = {}
        self.terms = []
        for t in prob.terms:
            fac = [(k, p) for k, p in t.pairs if p != 0]
            if len(fac) == 1 and fac[0][1] == 1 and fac[0][0] >= n:
                k = fac[0][0]
                m = t.C * _herm_multiplier(prob, k // n)
                key = (t.field, k % n)
                self.fold[t.field] = self.fold[t.field] or {}
                self.fold[t.field][k % n] = self.fold[t.field].get(k % n, 0) + m
                continue
            for k, _ in fac:
                if k >= n and k not in self.needed:
                    self.needed[k] = _herm_multiplier(prob, k // n)
            self.terms.append((t.field, t.C, fac))

    def __call__(self, t, y):
        prob, n = self.prob, self.prob.n
        axes = tuple(range(prob.ndim))
        U = y.reshape((n,) + tuple(prob.Ns))
        Uh = [sfft.rfftn(U[i], axes=axes, workers=self.workers) for i in range(n)]
        Y = {k: U[k] for k in range(n)}
        for k, m in self.needed.items():
            Y[k] = sfft.irfftn(m * Uh[k % n], s=prob.Ns, axes=axes, workers=self.workers)
        f = np.zeros((n,) + tuple(prob.Ns))
        for i in range(n):
            if self.fold[i]:
                acc = None
                for src, m in self.fold[i].items():
                    acc = m * Uh[src] if acc is None else acc + m * Uh[src]
                f[i] = sfft.irfftn(acc, s=prob.Ns, axes=axes, workers=self.workers)
        for field, C, fac in self.terms:
            prod = None
            for k, p in fac:
                v = Y[k] ** p if p > 0 else 1.0 / (Y[k] ** (-p))
                prod = v if prod is None else prod * v
            f[field] += C * (prod if prod is not None else 1.0)
        return f.reshape(-1)


def dp45_attempts(Ns: Sequence[int], Ls: Sequence[float], y: np.ndarray, h: float, attempts: int = 1,
                  workers: int = 1, rtol: float = 1e-8, atol: float = 1e-8) -> int:
    """Runs `attempts` DP45 attempts of the CGLE from state y; returns accepted steps."""
    prob = Problem(2, tuple(Ns), tuple(Ls), cgle_terms(len(Ns)))
    rhs = PortRHS(prob, workers)
    st = odp.DP45(y, atol, rtol, False, rhs)
    st.k[0] = rhs(0.0, st.y)
    t, acc = 0.0, 0
    for _ in range(attempts):
        ok, t, h = st.step(t, h, 0.0, np.inf)
        if ok:
            st.k[0] = st.k[6]
            acc += 1
    return acc
