"""Oracle: pseudospectral Y blocks and the dictionary RHS.

Test infrastructure only (see ``oracle/__init__``).  Restates reference ``rdcu.cu``:
``d1`` (rdcu.cu:78-99), ``make_term`` (rdcu.cu:101-106), the spectral branch of
``makeY`` (rdcu.cu:151-164) and ``dydt`` (rdcu.cu:167-184), with numpy's complex FFT in
place of cuFFT Z2Z.
"""
from __future__ import annotations

import numpy as np

from .problem import PI, Problem, pow_c


def freqs(N: int, L: float) -> np.ndarray:
    """Wavenumber of bin na along one axis, exactly as ``d1`` forms it (rdcu.cu:89-95):
    ``na*2*PI/L`` for na < N/2 (C integer division), else ``(na-N)*2*PI/L``.
    The Nyquist bin of an even N is kept with the negative sign."""
    na = np.arange(N)
    half = N // 2
    m = np.where(na < half, na * 2, (na - N) * 2).astype(np.float64)
    return m * PI / L


def d1(Yin: np.ndarray, axis: int, prob: Problem) -> np.ndarray:
    """``d1`` kernel (rdcu.cu:78-99): Yout = i*k_axis*Yin on the spectra of all n fields.
    ``Yin`` has shape (n, *Ns)."""
    k = freqs(prob.Ns[axis], prob.Ls[axis])
    shape = [1] * (prob.ndim + 1)
    shape[axis + 1] = prob.Ns[axis]
    k = k.reshape(shape)
    return (-k * Yin.imag) + 1j * (k * Yin.real)


def spectral_Y(y: np.ndarray, prob: Problem) -> np.ndarray:
    """All Y blocks, complex, shape (nY*n, N), index k = Yind*n + field.

    makeY spectral branch (rdcu.cu:151-164): forward FFT of the n fields; first
    derivative block 1+i = d1(yfft, i); second-derivative block j+i*ndim+ndim+1 =
    d1(block 1+i, j); inverse FFT of every block, scaled by 1/N.
    """
    n, ndim, Ns = prob.n, prob.ndim, tuple(prob.Ns)
    axes = tuple(range(1, ndim + 1))
    U = np.asarray(y, np.float64).reshape((n,) + Ns).astype(np.complex128)
    yfft = np.empty((prob.nY, n) + Ns, np.complex128)
    yfft[0] = np.fft.fftn(U, axes=axes)
    for i in range(ndim):
        yfft[1 + i] = d1(yfft[0], i, prob)
        for j in range(ndim):
            yfft[j + i * ndim + ndim + 1] = d1(yfft[1 + i], j, prob)
    # cuFFT's inverse is unnormalised and the reference scales by 1/N afterwards;
    # numpy's ifftn applies the same 1/N.
    Y = np.fft.ifftn(yfft, axes=tuple(a + 1 for a in axes))
    return Y.reshape(prob.nY * n, prob.N)


def dictionary_rhs(Yreal: np.ndarray, prob: Problem) -> np.ndarray:
    """``dydt`` accumulation (rdcu.cu:171-183): f = 0; for each term, term = 1, then
    ``term *= pow(Re Y_k, eta)`` per factor (make_term, rdcu.cu:101-106), then
    ``f[field] += C*term`` (cublasDaxpy).  ``Yreal`` has shape (nY*n, N)."""
    n, N = prob.n, prob.N
    f = np.zeros((n, N), np.float64)
    for term in prob.terms:
        tv = np.ones(N, np.float64)
        for (k, eta) in term.pairs:
            tv = tv * pow_c(Yreal[k], 1.0 * eta)
        f[term.field] = f[term.field] + term.C * tv
    return f.reshape(-1)


def rhs(y: np.ndarray, prob: Problem, return_Y: bool = False):
    """Pseudospectral ``dydt(t, y, f)`` (rdcu.cu:167-184).  Returns f (n*N,) and, if
    asked, the complex Y blocks (nY*n, N) that ``-D3`` writes to ``Y.dat``."""
    Y = spectral_Y(y, prob)
    f = dictionary_rhs(Y.real, prob)
    return (f, Y) if return_Y else f
