"""GPU: the discrete adjoint of fixed-step DP45 (rdcu_adjoint_forward/backward).

Checks, through the C ABI:
* duality with the oracle's tangent-linear model: <w, dyT> = <grad_y0, dy0> + <grad_C, dC>
  for random directions (relative 1e-9), on the CGLE and on random dictionaries with
  products of derivative blocks, in 1D, 2D and 3D, with odd and even grid sizes;
* central finite differences of the GPU forward map itself (relative 1e-6), for the
  initial condition and for every coupling coefficient;
* checkpoint spacing K does not change the result (bitwise);
* a recorded adaptive step sequence, torch.autograd.Function, coefficient replacement
  and the error paths.
"""
import numpy as np
import pytest

from oracle import tangent as otl
from oracle.problem import Problem, Term, cgle_terms
from tests.helpers import random_terms, rel_err, smooth_field, spec_terms

pytestmark = pytest.mark.gpu


def _solver(prob, fixed=True):
    import rdcu_b200 as R

    return R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), fixed=fixed)


def _grads(torch, s, y0, hs, K, w):
    y = torch.tensor(y0, dtype=torch.float64, device="cuda")
    yT = torch.empty_like(y)
    s.adjoint_forward(y.data_ptr(), hs, K, yT.data_ptr())
    lam = torch.tensor(w, dtype=torch.float64, device="cuda")
    g = torch.empty_like(y)
    gC = s.adjoint_backward(lam.data_ptr(), g.data_ptr())
    return yT.cpu().numpy(), g.cpu().numpy(), np.array(gC)


def _duality(prob, y0, hs, w, yT, gy, gC, rng, ndir=3):
    C = np.array([t.C for t in prob.terms])
    for _ in range(ndir):
        dy0 = smooth_field(rng, prob, amp=1.0) + 0.1 * rng.normal(size=y0.size)
        dC = rng.normal(size=C.size)
        yT_o, dyT = otl.dp45_tlm(y0, dy0, hs, prob, C, dC)
        assert rel_err(yT, yT_o) < 1e-10
        lhs = float(np.dot(w, dyT))
        rhs = float(np.dot(gy, dy0) + np.dot(gC, dC))
        assert abs(lhs - rhs) <= 1e-9 * max(abs(lhs), 1e-30), (lhs, rhs)


def _random_dictionary(rng, n, ndim, nterms, extra):
    """Random monomials plus fixed terms that cover every adjoint branch: an odd-order
    single derivative (folded; its transpose flips sign), a product of a derivative
    block with a field (derivative quantity in the pointwise VJP) and a constant."""
    return random_terms(rng, n, ndim, nterms, max_factors=2) + [Term(c, list(i)) for c, i in extra]


CASES = {
    "cgle2d": lambda rng: Problem(2, (32, 24), (40.0, 30.0), cgle_terms(2)),
    "cgle1d_odd": lambda rng: Problem(2, (45,), (30.0,), cgle_terms(1)),
    "cgle3d": lambda rng: Problem(2, (8, 6, 10), (10.0, 8.0, 12.0), cgle_terms(3)),
    # 128-point x rows: the forward stages run the fused inverse/forward x passes
    "cgle3d_rows": lambda rng: Problem(2, (4, 6, 128), (5.0, 6.0, 100.0), cgle_terms(3)),
    # 2D, n=2: Y index = Yind*2 + field; u0_x = 2, u1_y = 5, u0_xy = 8
    "random2d": lambda rng: Problem(2, (16, 15), (50.0, 45.0), _random_dictionary(
        rng, 2, 2, 7, [(0.7, [0, 2, 1]), (-0.4, [1, 2, 1, 0, 1]), (0.3, [0, 5, 1]), (0.2, [1, 8, 1, 1, 2]),
                       (0.5, [1])])),
    # 3D, n=1: u_x = 1, u_z = 3, u_xz = 6
    "random3d": lambda rng: Problem(1, (6, 4, 8), (12.0, 9.0, 15.0), _random_dictionary(
        rng, 1, 3, 6, [(0.6, [0, 3, 1]), (-0.5, [0, 1, 1, 0, 2]), (0.25, [0, 6, 1, 0, 1])])),
}
SEEDS = {"cgle2d": 1, "cgle1d_odd": 2, "cgle3d": 3, "random2d": 4, "random3d": 5, "cgle3d_rows": 6}


@pytest.mark.parametrize("case", sorted(CASES))
def test_duality_with_tangent_linear_model(cuda, case):
    rng = np.random.default_rng(SEEDS[case])
    prob = CASES[case](rng)
    y0 = smooth_field(rng, prob, amp=0.5)
    h = 1e-2 if case.startswith("cgle") else 2e-3
    hs = [h] * 11
    w = rng.normal(size=y0.size)
    s = _solver(prob)
    yT, gy, gC = _grads(cuda, s, y0, hs, 4, w)
    _duality(prob, y0, hs, w, yT, gy, gC, rng)
    s.close()


def test_central_differences_on_the_gpu_map(cuda):
    """dL/dy0 and every dL/dC_t against central differences of the GPU forward map,
    L = <w, yT>, relative 1e-6."""
    rng = np.random.default_rng(3)
    prob = Problem(2, (32, 32), (40.0, 40.0), cgle_terms(2))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    hs = [5e-3] * 30
    w = rng.normal(size=y0.size)
    s = _solver(prob)
    _, gy, gC = _grads(cuda, s, y0, hs, 7, w)
    C = np.array([t.C for t in prob.terms])

    def L(yy, CC):
        s.set_coefficients(list(CC))
        yd = cuda.tensor(yy, dtype=cuda.float64, device="cuda")
        out = cuda.empty_like(yd)
        s.adjoint_forward(yd.data_ptr(), hs, 1000, out.data_ptr())
        return float(np.dot(w, out.cpu().numpy()))

    for _ in range(2):
        d = rng.normal(size=y0.size)
        eps = 1e-5
        fd = (L(y0 + eps * d, C) - L(y0 - eps * d, C)) / (2 * eps)
        assert abs(fd - float(np.dot(gy, d))) <= 1e-6 * abs(fd)
    for t in range(C.size):
        eps = 1e-5 * max(1.0, abs(C[t]))
        Cp, Cm = C.copy(), C.copy()
        Cp[t] += eps
        Cm[t] -= eps
        fd = (L(y0, Cp) - L(y0, Cm)) / (2 * eps)
        assert abs(fd - gC[t]) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(gC))), (t, fd, gC[t])
    s.close()


def test_checkpoint_spacing_is_bitwise_neutral(cuda):
    rng = np.random.default_rng(8)
    prob = Problem(2, (24, 16), (20.0, 15.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.5)
    hs = [1e-2] * 12
    w = rng.normal(size=y0.size)
    s = _solver(prob)
    ref = _grads(cuda, s, y0, hs, 12, w)
    for K in (1, 5, 7):
        got = _grads(cuda, s, y0, hs, K, w)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b)
    s.close()


def test_recorded_adaptive_sequence(cuda):
    """Replay of the accepted steps of an adaptive run: the final state equals the
    adaptive run's (the stage arithmetic is shared) and the adjoint passes duality."""
    import rdcu_b200 as R
    from rdcu_b200.adjoint import accepted_steps

    rng = np.random.default_rng(4)
    prob = Problem(2, (32, 24), (40.0, 30.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.5)
    a = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), rtol=1e-6, atol=1e-6)
    yd = cuda.tensor(y0, dtype=cuda.float64, device="cuda")
    cuda.cuda.synchronize()
    hs = accepted_steps(a, yd.data_ptr(), 0.0, 1e-3, 0.3)
    assert len(hs) > 3 and len(set(hs)) > 1
    yA = cuda.empty_like(yd)
    a.get_state(yA.data_ptr())
    w = rng.normal(size=y0.size)
    s = _solver(prob)
    yT, gy, gC = _grads(cuda, s, y0, hs, 3, w)
    assert rel_err(yT, yA.cpu().numpy()) < 1e-13
    _duality(prob, y0, hs, w, yT, gy, gC, rng, ndir=2)
    a.close()
    s.close()


def test_autograd_function(cuda):
    from rdcu_b200.adjoint import integrate

    torch = cuda
    rng = np.random.default_rng(9)
    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.5)
    s = _solver(prob)
    hs = [1e-2] * 9
    y = torch.tensor(y0, dtype=torch.float64, device="cuda", requires_grad=True)
    C = torch.tensor([t.C for t in prob.terms], dtype=torch.float64, requires_grad=True)
    yT = integrate(s, y, C, hs, K=4)
    loss = (yT ** 2).sum() + yT[: prob.N].sum()
    loss.backward()
    gy, gC = y.grad.cpu().numpy(), C.grad.numpy()
    # same gradient through the raw ABI with lambda = dloss/dyT
    lam = 2 * yT.detach().cpu().numpy()
    lam[: prob.N] += 1
    _, gy2, gC2 = _grads(torch, s, y0, hs, 4, lam)
    assert np.array_equal(gy, gy2) and np.allclose(gC, gC2, rtol=0, atol=0)
    # a second forward before backward: the Function re-records its own forward
    y_b = torch.tensor(y0, dtype=torch.float64, device="cuda", requires_grad=True)
    yT1 = integrate(s, y_b, C.detach(), hs, K=4)
    _ = integrate(s, torch.tensor(y0[::-1].copy(), dtype=torch.float64, device="cuda"), C.detach(), hs, K=4)
    (yT1 ** 2).sum().backward()
    lam = 2 * yT1.detach().cpu().numpy()
    _, gy3, _ = _grads(torch, s, y0, hs, 4, lam)
    assert np.array_equal(y_b.grad.cpu().numpy(), gy3)
    s.close()


def test_set_coefficients_matches_a_fresh_handle(cuda):
    rng = np.random.default_rng(12)
    prob = Problem(2, (16, 12), (9.0, 7.0), random_terms(rng, 2, 2, 8, max_factors=2))
    y0 = smooth_field(rng, prob, amp=0.5)
    C2 = rng.normal(size=len(prob.terms))
    prob2 = Problem(2, prob.Ns, prob.Ls, [type(t)(float(c), list(t.ints)) for t, c in zip(prob.terms, C2)])
    s, s2 = _solver(prob), _solver(prob2)
    s.set_coefficients(list(C2))
    y = cuda.tensor(y0, dtype=cuda.float64, device="cuda")
    f1, f2 = cuda.empty_like(y), cuda.empty_like(y)
    cuda.cuda.synchronize()
    s.rhs(y.data_ptr(), f1.data_ptr())
    s2.rhs(y.data_ptr(), f2.data_ptr())
    assert cuda.equal(f1, f2)
    s.close()
    s2.close()


def test_error_paths(cuda):
    import rdcu_b200 as R

    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y = cuda.zeros(2 * prob.N, dtype=cuda.float64, device="cuda")
    a = _solver(prob, fixed=False)
    with pytest.raises(R.RdcuError) as e:
        a.adjoint_forward(y.data_ptr(), [1e-2], 1)
    assert e.value.code == R.RDCU_ERR_STATE
    s = _solver(prob)
    with pytest.raises(R.RdcuError) as e:
        s.adjoint_backward(y.data_ptr(), y.data_ptr())
    assert e.value.code == R.RDCU_ERR_STATE
    with pytest.raises(R.RdcuError) as e:
        s.adjoint_forward(y.data_ptr(), [1e-2, -1.0], 1)
    assert e.value.code == R.RDCU_ERR_INVALID
    b = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), method=R.METHOD_BDF)
    with pytest.raises(R.RdcuError) as e:
        b.set_coefficients([1.0] * len(prob.terms))
    assert e.value.code == R.RDCU_ERR_UNSUPPORTED
    for x in (a, s, b):
        x.close()


def test_long_segments_and_step_sequences(cuda):
    """Segments longer than the controller's attempt log (4096) and a non-uniform step
    sequence (direct launches): K = nsteps and K = 1000 agree bitwise."""
    rng = np.random.default_rng(17)
    prob = Problem(2, (8, 8), (10.0, 10.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.5)
    hs = [1e-4 * (1.0 + 0.1 * (j % 3)) for j in range(4200)]
    w = rng.normal(size=y0.size)
    s = _solver(prob)
    a = _grads(cuda, s, y0, hs, 4200, w)
    b = _grads(cuda, s, y0, hs, 1000, w)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    s.close()
