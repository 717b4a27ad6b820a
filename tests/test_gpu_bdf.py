"""GPU parity: the finite-difference RHS, CSR Jacobian and BDF integrator of librdcu
against the oracle (restatements of rdcu.cu:122-149,186-250,385-596 and bdf.cu).

The oracle's BDF solves A dd = b with a direct sparse LU (as the reference's cuDSS
does); the library uses preconditioned GMRES to a 1e-12 relative residual.  Short runs
must give the same accepted-step count, the same order sequence and states within
1e-8 relative.
"""
import tempfile

import numpy as np
import pytest

from oracle import fd as ofd
from oracle import run as orun
from oracle.problem import Problem, brusselator_coupling_lines, cgle_terms, parse_term
from tests.helpers import five_field_stiff_problem, rel_err, random_terms, spec_terms

pytestmark = pytest.mark.gpu


def _solver(prob, **kw):
    import rdcu_b200 as R

    return R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), method=R.METHOD_BDF, **kw)


@pytest.mark.parametrize("Ns", [(12,), (8, 6), (5, 7), (4, 5, 6), (6, 6, 4)])
def test_fd_rhs_and_jacobian_random(cuda, Ns):
    rng = np.random.default_rng(sum(Ns) + 100 * len(Ns))
    n, ndim = 2, len(Ns)
    Ls = tuple(float(rng.uniform(1, 5)) for _ in Ns)
    prob = Problem(n, Ns, Ls, random_terms(rng, n, ndim, 10))
    y = rng.uniform(0.5, 1.5, n * prob.N)
    s = _solver(prob)
    f = np.empty_like(y)
    Y = np.empty(prob.nY * n * prob.N * 2)
    s.rhs(y.ctypes.data, f.ctypes.data, Y.ctypes.data)
    assert rel_err(f, ofd.rhs(y, prob)) < 1e-12
    Yo = ofd.fd_Y(y, prob)
    Yc = Y.view(np.complex128).reshape(prob.nY * n, prob.N)
    assert rel_err(Yc.real, Yo) < 1e-12 and np.all(Yc.imag == 0)
    nnz_max = s.info().nnz_max
    rows = np.empty(n * prob.N + 1, np.int32)
    cols = np.empty(max(1, nnz_max), np.int32)
    vals = np.empty(max(1, nnz_max))
    nnz = s.jac(y.ctypes.data, rows.ctypes.data, cols.ctypes.data, vals.ctypes.data)
    r0, c0, v0 = ofd.jacobian(y, prob)
    assert nnz == len(c0)
    np.testing.assert_array_equal(rows, r0)
    np.testing.assert_array_equal(cols[:nnz], c0)
    assert rel_err(vals[:nnz], v0) < 1e-12
    s.close()


def _bdf_run(prob, y0, t1, dt, rtol):
    import rdcu_b200 as R

    s = _solver(prob, rtol=rtol, atol=rtol)
    y = np.array(y0)
    h0 = dt / 100
    s.set_state(0.0, h0, y.ctypes.data)
    t_eval = [dt * k for k in range(1, int(t1 / dt) + 1)]
    ev = {"h": [], "acc": [], "states": [], "order": []}

    def cb(e):
        if e.kind == R.EV_ATTEMPT:
            ev["h"].append(e.h)
            ev["acc"].append(e.accepted)
            ev["order"].append(e.order)
        elif e.kind == R.EV_EVAL:
            ev["states"].append(s.copy_to_numpy(e.y, prob.n * prob.N))
        return 0

    s.solve(t1, t_eval, callback=cb)
    s.close()
    return ev


@pytest.mark.parametrize("case", ["bruss16", "cgle16", "bruss3d"])
def test_bdf_matches_oracle(cuda, case):
    if case == "bruss16":
        prob = Problem(2, (16, 16), (16.0, 16.0), [parse_term(s) for s in brusselator_coupling_lines()])
        rng = np.random.default_rng(3)
        y0 = np.concatenate([1.0 + 0.1 * rng.uniform(-1, 1, prob.N), 3.0 + 0.1 * rng.uniform(-1, 1, prob.N)])
        t1, dt, rtol = 2.0, 0.5, 1e-6
    elif case == "cgle16":
        prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
        y0 = np.random.default_rng(4).uniform(-1, 1, 2 * prob.N)
        t1, dt, rtol = 0.5, 0.25, 1e-6
    else:
        terms = ["1.0,0", "-4.0,0,0,1", "1.0,0,0,2,1,1", "1.0,0,%d,1", "3.0,1,0,1", "-1.0,1,0,2,1,1", "8.0,1,%d,1"]
        # laplacians in 3D: u0_aa = 2 + 6 + 8a, u1_aa = 9 + 8a
        lines = terms[:3] + ["1.0,0,%d,1" % (8 + 8 * a) for a in range(3)] + terms[4:6] + \
            ["8.0,1,%d,1" % (9 + 8 * a) for a in range(3)]
        prob = Problem(2, (6, 8, 6), (6.0, 8.0, 6.0), [parse_term(s) for s in lines])
        rng = np.random.default_rng(5)
        y0 = np.concatenate([1.0 + 0.1 * rng.uniform(-1, 1, prob.N), 3.0 + 0.1 * rng.uniform(-1, 1, prob.N)])
        t1, dt, rtol = 1.0, 0.5, 1e-6
    ev = _bdf_run(prob, y0, t1, dt, rtol)
    # oracle: the reference driver loop with SuperLU
    with tempfile.TemporaryDirectory() as wd:
        fb = wd + "/o"
        y0.tofile(fb + "ic.dat")
        cfg = orun.RunConfig(n=2, Ns=prob.Ns, Ls=prob.Ls, terms=prob.terms, t1=t1, dt=dt, rtol=rtol, atol=rtol,
                             stiff=True)
        summ = orun.run(fb, cfg)
        oh = np.fromfile(fb + "steps.dat")
        ost = np.fromfile(fb + "states.dat").reshape(-1, 2 * prob.N)[1:]
    assert sum(ev["acc"]) == summ["steps"]
    assert len(ev["h"]) == len(oh)
    assert np.max(np.abs(np.array(ev["h"]) - oh) / np.abs(oh)) < 1e-8
    assert len(ev["states"]) == len(ost)
    for a, b in zip(ev["states"], ost):
        assert rel_err(a, b) < 1e-8


def test_unpreconditioned_gmres_with_restarts(cuda):
    """Five fields, one more than the preconditioner's n x n mode solves take, so the
    linear solves run plain GMRES(40); on this stiff diffusion system (condition ~100)
    most solves need several restart cycles to reach the 1e-12 relative residual.  The
    run must match the direct-solve oracle step for step, as the preconditioned runs do,
    and its solver counts must match the oracle's restatement of the same GMRES."""
    import rdcu_b200 as R

    prob, y0 = five_field_stiff_problem()
    n = prob.n
    t1, dt, rtol = 1.0, 0.5, 1e-4
    s = _solver(prob, rtol=rtol, atol=rtol)
    y = np.array(y0)  # the library reads the state from this buffer
    s.set_state(0.0, dt / 100, y.ctypes.data)
    ev = {"h": [], "acc": [], "states": []}

    def cb(e):
        if e.kind == R.EV_ATTEMPT:
            ev["h"].append(e.h)
            ev["acc"].append(e.accepted)
        elif e.kind == R.EV_EVAL:
            ev["states"].append(s.copy_to_numpy(e.y, n * prob.N))
        return 0

    s.solve(t1, [dt, 2 * dt], callback=cb)
    iters, solves, cycles = s.linear_stats()
    s.close()
    assert solves > 0 and cycles > solves and iters > 40 * (cycles - solves)
    out = {}
    for linear in ("lu", "gmres"):
        with tempfile.TemporaryDirectory() as wd:
            fb = wd + "/o"
            y0.tofile(fb + "ic.dat")
            cfg = orun.RunConfig(n=n, Ns=prob.Ns, Ls=prob.Ls, terms=prob.terms, t1=t1, dt=dt, rtol=rtol,
                                 atol=rtol, stiff=True, linear=linear)
            summ = orun.run(fb, cfg)
            out[linear] = (summ, np.fromfile(fb + "steps.dat"),
                           np.fromfile(fb + "states.dat").reshape(-1, n * prob.N)[1:])
    summ, oh, ost = out["lu"]
    assert sum(ev["acc"]) == summ["steps"]
    assert len(ev["h"]) == len(oh)
    assert np.max(np.abs(np.array(ev["h"]) - oh) / np.abs(oh)) < 1e-8
    assert len(ev["states"]) == len(ost)
    for a, b in zip(ev["states"], ost):
        assert rel_err(a, b) < 1e-8
    st = out["gmres"][0]["linear"]
    assert solves == st["solves"]
    assert abs(iters - st["iterations"]) <= 0.02 * st["iterations"]
    assert abs(cycles - st["cycles"]) <= 0.02 * st["cycles"]


def test_linear_stats_of_a_dp45_handle_are_zero(cuda):
    import rdcu_b200 as R

    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob))
    assert s.linear_stats() == (0, 0, 0)
    s.close()
