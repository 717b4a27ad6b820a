"""Oracle: finite-difference stencils, FD Y blocks and the analytic CSR Jacobian.

Test infrastructure only (see ``oracle/__init__``).  Restates reference ``rdcu.cu``:
``init_dY`` (rdcu.cu:385-596), the finite-difference branch of ``makeY``
(rdcu.cu:122-149), ``jac`` (rdcu.cu:186-250) with ``make_jac_term`` (rdcu.cu:108-115),
and the csrgeam2 union/sum semantics the reference relies on.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .problem import Problem, pow_c


def _ravel(ns, Ns) -> int:
    j = 0
    stride = 1
    for d in range(len(Ns) - 1, -1, -1):
        j += ns[d] * stride
        stride *= Ns[d]
    return j


def _unravel(j, Ns) -> List[int]:
    ns = [0] * len(Ns)
    stride = 1
    for d in range(len(Ns) - 1, -1, -1):
        ns[d] = (j // stride) % Ns[d]
        stride *= Ns[d]
    return ns


def stencils(prob: Problem):
    """COO stencil per Y block (rows, cols, vals), each row's entries sorted by column as
    ``qsort_r`` leaves them (rdcu.cu:449,508,569).  Block 0 is the identity, block 1+a is
    d_a (+-0.5/dx_a), block b + a*ndim + ndim + 1 is d_a d_b: (1,-2,1)/dx_a^2 when a == b,
    else (+0.5,-0.5,-0.5,+0.5)/(dx_a dx_b) at (--,-+,+-,++) -- twice the textbook 1/4
    mixed stencil, reproduced as the reference has it."""
    Ns, Ls, ndim, N = list(prob.Ns), list(prob.Ls), prob.ndim, prob.N
    out = [None] * prob.nY
    idx = np.arange(N)
    out[0] = (idx.copy(), idx.copy(), np.ones(N))
    for axis in range(ndim):
        rows, cols, vals = [], [], []
        scale = Ls[axis] / Ns[axis]
        for j in range(N):
            ns = _unravel(j, Ns)
            ns[axis] = (ns[axis] + 1) % Ns[axis]
            jp = _ravel(ns, Ns)
            ns[axis] = (ns[axis] + Ns[axis] - 2) % Ns[axis]
            jm = _ravel(ns, Ns)
            ent = sorted([(jm, -0.5 / scale, 0), (jp, 0.5 / scale, 1)], key=lambda e: e[0])
            for c, v, _ in ent:
                rows.append(j); cols.append(c); vals.append(v)
        out[axis + 1] = (np.array(rows), np.array(cols), np.array(vals))
        for axis2 in range(ndim):
            Yind = axis2 + ndim * axis + ndim + 1
            rows, cols, vals = [], [], []
            scale = (Ls[axis] / Ns[axis]) * (Ls[axis2] / Ns[axis2])
            for j in range(N):
                ns = _unravel(j, Ns)
                ns[axis] = (ns[axis] + 1) % Ns[axis]
                jp = _ravel(ns, Ns)
                ns[axis] = (ns[axis] + Ns[axis] - 2) % Ns[axis]
                jm = _ravel(ns, Ns)
                ns[axis] = (ns[axis] + 1) % Ns[axis]
                if axis == axis2:
                    ent = [(jm, 1.0 / scale), (j, -2.0 / scale), (jp, 1.0 / scale)]
                else:
                    ns[axis] = (ns[axis] + 1) % Ns[axis]
                    ns[axis2] = (ns[axis2] + 1) % Ns[axis2]
                    jpp = _ravel(ns, Ns)
                    ns[axis2] = (ns[axis2] + Ns[axis2] - 2) % Ns[axis2]
                    jpm = _ravel(ns, Ns)
                    ns[axis] = (ns[axis] + Ns[axis] - 2) % Ns[axis]
                    jmm = _ravel(ns, Ns)
                    ns[axis2] = (ns[axis2] + 2) % Ns[axis2]
                    jmp = _ravel(ns, Ns)
                    ent = [(jmm, 0.5 / scale), (jmp, -0.5 / scale), (jpm, -0.5 / scale),
                           (jpp, 0.5 / scale)]
                ent = sorted(ent, key=lambda e: e[0])
                for c, v in ent:
                    rows.append(j); cols.append(c); vals.append(v)
            out[Yind] = (np.array(rows), np.array(cols), np.array(vals))
    return out


def _coo_matvec(st, x: np.ndarray, N: int) -> np.ndarray:
    rows, cols, vals = st
    out = np.zeros(N, np.float64)
    np.add.at(out, rows, vals * x[cols])
    return out


def fd_Y(y: np.ndarray, prob: Problem, st=None) -> np.ndarray:
    """Real Y blocks (nY*n, N) of the FD branch of makeY (rdcu.cu:119,122-149):
    block 0 is a copy of y, block Yind of field i is D_Yind @ y_i (cusparseSpMV)."""
    if st is None:
        st = stencils(prob)
    n, N = prob.n, prob.N
    y = np.asarray(y, np.float64).reshape(n, N)
    Y = np.empty((prob.nY * n, N), np.float64)
    Y[:n] = y
    for Yind in range(1, prob.nY):
        for i in range(n):
            Y[Yind * n + i] = _coo_matvec(st[Yind], y[i], N)
    return Y


def rhs(y: np.ndarray, prob: Problem, st=None) -> np.ndarray:
    """FD ``dydt`` (rdcu.cu:167-184 with the FD makeY)."""
    from .spectral import dictionary_rhs

    return dictionary_rhs(fd_Y(y, prob, st), prob)


def jacobian(y: np.ndarray, prob: Problem, st=None) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """CSR Jacobian (rows n*N+1, cols, vals) as ``jac`` builds it (rdcu.cu:186-250).

    For each term i and factor j (in order), the values are
    ``C*eta_j * prod_k pow(Y_k, eta_k - [k==j])`` per point -- evaluated in the
    reference's order: term = 1; for each factor k: (if k == j: term *= C*eta_k) then
    term *= pow(Y_k, eta_k - [k==j]) -- times the stencil of Y block c[i][j]/n, placed
    at block (field, c[i][j] % n).  The contributions are summed as csrgeam2 does:
    pattern = sorted union of columns per row, explicit zeros kept, values
    accumulated in term/factor order.
    """
    if st is None:
        st = stencils(prob)
    n, N = prob.n, prob.N
    Yr = fd_Y(y, prob, st)
    nrow = n * N
    acc = [dict() for _ in range(nrow)]
    for term in prob.terms:
        pairs = term.pairs
        for jf, (kj, _pj) in enumerate(pairs):
            tv = np.ones(N, np.float64)
            for kf, (kk, pk) in enumerate(pairs):
                pw = pk
                if kf == jf:
                    tv = (term.C * pw) * tv
                    pw -= 1
                tv = tv * pow_c(Yr[kk], 1.0 * pw)
            dYind = kj // n
            rows, cols, vals = st[dYind]
            rowoff = N * term.field
            coloff = N * (kj % n)
            v = vals * tv[rows]
            for r, c, val in zip(rows + rowoff, cols + coloff, v):
                d = acc[r]
                d[c] = (d[c] + val) if c in d else val
    rowptr = np.zeros(nrow + 1, np.int32)
    cols_out, vals_out = [], []
    for r in range(nrow):
        items = sorted(acc[r].items())
        rowptr[r + 1] = rowptr[r] + len(items)
        for c, v in items:
            cols_out.append(c); vals_out.append(v)
    return rowptr, np.array(cols_out, np.int32), np.array(vals_out, np.float64)


def csr_to_scipy(rowptr, cols, vals, nrow):
    import scipy.sparse as sp

    return sp.csr_matrix((vals, cols, rowptr), shape=(nrow, nrow))
