"""The oracle's tangent-linear DP45 (the checker of the GPU adjoint) against central
finite differences of the oracle's own fixed-step DP45 (CPU)."""
import numpy as np
import pytest

from oracle import tangent as otl
from oracle.problem import Problem, Term, cgle_terms
from tests.helpers import random_terms, smooth_field


def _fd(fun, x, d, eps):
    return (fun(x + eps * d) - fun(x - eps * d)) / (2 * eps)


@pytest.mark.parametrize("case", ["cgle2d", "random1d", "random3d"])
def test_tlm_matches_central_differences(case):
    rng = np.random.default_rng(5)
    if case == "cgle2d":
        prob = Problem(2, (8, 6), (10.0, 7.0), cgle_terms(2))
    elif case == "random1d":
        prob = Problem(2, (10,), (6.0,), random_terms(rng, 2, 1, 7, max_factors=2))
    else:
        prob = Problem(1, (4, 6, 5), (3.0, 4.0, 5.0), random_terms(rng, 1, 3, 6, max_factors=2))
    y0 = smooth_field(rng, prob, amp=0.3)
    dy0 = smooth_field(rng, prob, amp=1.0)
    C = np.array([t.C for t in prob.terms])
    dC = rng.normal(size=C.size)
    hs = [2e-3, 1e-3, 3e-3, 2e-3]
    _, dyT = otl.dp45_tlm(y0, dy0, hs, prob, C, dC)
    # joint direction in (y0, C)
    fd = _fd(lambda s: otl.dp45_fixed(y0 + s * dy0, hs, prob, C + s * dC), 0.0, 1.0, 1e-5)
    assert np.max(np.abs(dyT - fd)) <= 1e-7 * max(1.0, np.max(np.abs(dyT)))


def test_rhs_jvp_linear_in_coefficients():
    rng = np.random.default_rng(2)
    prob = Problem(2, (6, 4), (5.0, 3.0), [Term(1.5, [0, 2, 1, 1, 2]), Term(-0.5, [1, 0, 3]), Term(2.0, [1])])
    y = smooth_field(rng, prob)
    dC = np.array([1.0, 0.0, 0.0])
    df = otl.rhs_jvp(y, np.zeros_like(y), prob, None, dC)
    # d f / d C_0 = the first monomial u_x * v^2 ... evaluated directly
    from oracle import spectral as osp

    Q = osp.spectral_Y(y, prob).real
    expect = np.zeros((2, prob.N))
    expect[0] = Q[2] * Q[1] ** 2
    assert np.max(np.abs(df - expect.ravel())) < 1e-12
