"""Shared helpers for the parity tests (CPU side: problem generators, comparisons)."""
from __future__ import annotations

import numpy as np

from oracle.problem import Problem, Term, parse_term


def rel_err(a, b) -> float:
    """max|a-b| / max|b| (max-norm relative difference)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / max(den, 1e-300) if a.size else 0.0


def random_terms(rng, n: int, ndim: int, nterms: int, max_factors: int = 3, deriv: bool = True,
                 allow_zero_pow: bool = True) -> list:
    """Random dictionary: coefficients N(0,1), factors over all Y indices (or fields only),
    powers 0..3 (power 0 allowed), constant terms included."""
    nY = 1 + ndim + ndim * ndim
    out = []
    for _ in range(nterms):
        field = int(rng.integers(0, n))
        nf = int(rng.integers(0, max_factors + 1))
        ints = [field]
        for _ in range(nf):
            k = int(rng.integers(0, nY * n)) if deriv else int(rng.integers(0, n))
            p = int(rng.integers(0 if allow_zero_pow else 1, 4))
            ints += [k, p]
        out.append(Term(float(rng.normal()), ints))
    return out


def smooth_field(rng, prob: Problem, amp: float = 1.0, modes: int = 3) -> np.ndarray:
    """Sum of a few random low Fourier modes per field (plus an offset)."""
    grids = np.meshgrid(*[np.arange(N) / N for N in prob.Ns], indexing="ij")
    out = []
    for _ in range(prob.n):
        u = np.full(prob.Ns, float(rng.normal()))
        for _ in range(modes):
            k = [int(rng.integers(-2, 3)) for _ in prob.Ns]
            ph = float(rng.uniform(0, 2 * np.pi))
            arg = sum(2 * np.pi * kk * g for kk, g in zip(k, grids))
            u = u + amp * float(rng.normal()) * np.cos(arg + ph)
        out.append(u.ravel())
    return np.concatenate(out)


def spec_terms(prob: Problem):
    return [(t.C, list(t.ints)) for t in prob.terms]


def defect_state(Ns, seed: int, frame: int = 0, nterms: int = 3, noise: float = 0.1, drift: float = 1.0):
    """A 2-field state (u block, v block) whose phase carries vortex lines: each term adds
    atan2(sin(2 pi (x_b - q)/N_b), sin(2 pi (x_a - p)/N_a)) -- four periodic lines along the
    third axis, wobbling along it and drifting with the frame index -- plus phase noise.
    Same seed, later frame: the same lines moved on."""
    rng = np.random.default_rng(seed)
    Ns = tuple(int(n) for n in Ns)
    g = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in Ns], indexing="ij")
    th = np.zeros(Ns)
    for _ in range(nterms):
        ax = int(rng.integers(3))
        a, b = [x for x in range(3) if x != ax]
        p0, q0 = rng.uniform(0, Ns[a]), rng.uniform(0, Ns[b])
        vp, vq = rng.normal(size=2) * drift
        amp, ph = rng.uniform(0, 2.5), rng.uniform(0, 2 * np.pi)
        s = 2 * np.pi * g[ax] / Ns[ax] + ph
        p = p0 + vp * frame + amp * np.sin(s)
        q = q0 + vq * frame + amp * np.cos(s)
        th += np.arctan2(np.sin(2 * np.pi * (g[b] - q) / Ns[b]), np.sin(2 * np.pi * (g[a] - p) / Ns[a]))
    th += noise * np.random.default_rng([seed, frame]).normal(size=Ns)
    r = 1.0 + 0.2 * np.random.default_rng([seed, frame, 1]).uniform(size=Ns)
    return np.concatenate([(r * np.cos(th)).ravel(), (r * np.sin(th)).ravel()])


def five_field_stiff_problem():
    """A stiff system of five coupled diffusing fields on an 8 x 8 periodic grid, L = 8:
    u_f' = D_f (d00 + d11) u_f - u_f + 0.5 u_{f+1} - 0.2 u_f^3, D = 10, 20, 40, 80, 5
    (d00 u_f = Y[15+f], d11 u_f = Y[30+f] for n = 5).  Five fields are beyond the BDF
    preconditioner, and at rtol = 1e-4 the late steps (h ~ 0.15) make GMRES(40) restart.
    Returns the problem and the initial state, U[0.5, 1.5] with numpy seed 6."""
    n = 5
    D = [10.0, 20.0, 40.0, 80.0, 5.0]
    lines = []
    for f in range(n):
        lines += ["%g,%d,%d,1" % (D[f], f, 15 + f), "%g,%d,%d,1" % (D[f], f, 30 + f), "-1.0,%d,%d,1" % (f, f),
                  "0.5,%d,%d,1" % (f, (f + 1) % n), "-0.2,%d,%d,3" % (f, f)]
    prob = Problem(n, (8, 8), (8.0, 8.0), [parse_term(s) for s in lines])
    return prob, np.random.default_rng(6).uniform(0.5, 1.5, n * prob.N)
