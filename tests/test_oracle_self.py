"""Self-consistency of the oracle (CPU): analytic derivatives, the Hermitian form of
the reference's multipliers, the FD Jacobian against finite differences of the FD RHS,
the convergence orders of the DP45 and BDF restatements, the CPU port, and the BDF with
the library's GMRES solver against the direct solve."""
import tempfile

import numpy as np
import pytest

from oracle import bdf as obdf
from oracle import cpu_port
from oracle import dp45 as odp
from oracle import fd as ofd
from oracle import run as orun
from oracle import spectral as osp
from oracle.problem import Problem, cgle_terms, parse_term
from tests.helpers import five_field_stiff_problem, random_terms, rel_err


def _grid(prob):
    return np.meshgrid(*[np.arange(N) * (L / N) for N, L in zip(prob.Ns, prob.Ls)], indexing="ij")


def test_spectral_derivatives_of_a_plane_wave():
    prob = Problem(1, (12, 10), (3.0, 5.0), [])
    X, Y = _grid(prob)
    k0, k1 = 2 * np.pi / 3.0 * 2, 2 * np.pi / 5.0 * 3
    u = np.sin(k0 * X + k1 * Y)
    Yb = osp.spectral_Y(u.ravel(), prob).real.reshape(prob.nY, *prob.Ns)
    c = np.cos(k0 * X + k1 * Y)
    assert np.max(np.abs(Yb[1] - k0 * c)) < 1e-12
    assert np.max(np.abs(Yb[2] - k1 * c)) < 1e-12
    assert np.max(np.abs(Yb[3] + k0 * k0 * u)) < 1e-11   # u_00
    assert np.max(np.abs(Yb[4] + k0 * k1 * u)) < 1e-11   # u_01
    assert np.max(np.abs(Yb[6] + k1 * k1 * u)) < 1e-11   # u_11


@pytest.mark.parametrize("Ns", [(8,), (7,), (6, 8), (5, 4), (4, 6, 3)])
def test_hermitian_multipliers_reproduce_real_part(Ns):
    """Re(IFFT(M U)) of the reference's full complex transform equals the real-to-complex
    form with (M(k) + conj(M(-k)))/2, including its Nyquist conventions and the
    (na - N) map for odd N."""
    rng = np.random.default_rng(len(Ns))
    prob = Problem(1, Ns, tuple(float(rng.uniform(1, 4)) for _ in Ns), [])
    u = rng.uniform(-1, 1, prob.N)
    Yb = osp.spectral_Y(u, prob).real
    import scipy.fft as sfft

    Uh = sfft.rfftn(u.reshape(Ns))
    for yind in range(prob.nY):
        m = cpu_port._herm_multiplier(prob, yind)
        got = sfft.irfftn(m * Uh, s=Ns).ravel()
        assert np.max(np.abs(got - Yb[yind])) <= 1e-12 * max(1.0, np.max(np.abs(Yb[yind]))), yind


def test_fd_jacobian_matches_finite_differences():
    rng = np.random.default_rng(7)
    prob = Problem(2, (6, 5), (3.0, 4.0), random_terms(rng, 2, 2, 8, allow_zero_pow=False))
    y = rng.uniform(0.5, 1.5, prob.n * prob.N)
    v = rng.normal(size=y.size)
    rows, cols, vals = ofd.jacobian(y, prob)
    J = ofd.csr_to_scipy(rows, cols, vals, y.size)
    eps = 1e-6
    fd = (ofd.rhs(y + eps * v, prob) - ofd.rhs(y - eps * v, prob)) / (2 * eps)
    assert rel_err(J @ v, fd) < 1e-7


def test_dp45_fifth_order_on_linear_decay():
    lam = -2.0
    errs = []
    for h in (0.1, 0.05):
        st = odp.DP45(np.array([1.0]), 1e-8, 1e-8, True, lambda t, y: lam * y)
        st.k[0] = st.dydt(0, st.y)
        t = 0.0
        for _ in range(int(round(1.0 / h))):
            ok, t, _ = st.step(t, h, 0, np.inf)
            st.k[0] = st.k[6]
        errs.append(abs(st.y[0] - np.exp(lam)))
    assert 25 < errs[0] / errs[1] < 40  # ~2^5


def test_bdf_linear_stiff_problem_accuracy():
    # du/dt = -50 (u - cos t): smooth solution after a fast transient
    lam = -50.0
    prob_jac = lambda t, y: (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([lam]))
    st = obdf.BDF([np.array([0.0])], 0, 1e-8, 1e-6, False, lambda t, y: lam * (y - np.cos(t)), prob_jac)
    # the RHS depends on t: the restatement passes t + h, as bdf.cu does
    t, h = 0.0, 1e-4
    st.setup(t, h)
    while t < 2.0:
        ok, t, h = st.step(t, h, 0.0, np.inf)
    exact_like = (lam * lam * np.cos(t) - lam * np.sin(t)) / (lam * lam + 1)
    assert abs(st.D[0][0] - exact_like) < 1e-4
    assert 1 <= st.order <= 5


def test_cpu_port_equals_oracle_rhs():
    rng = np.random.default_rng(0)
    for Ns in [(16, 12), (8, 6, 10), (12,)]:
        prob = Problem(2, Ns, tuple(10.0 + i for i in range(len(Ns))), cgle_terms(len(Ns)))
        y = rng.uniform(-1, 1, 2 * prob.N)
        assert rel_err(cpu_port.PortRHS(prob, 2)(0, y), osp.rhs(y, prob)) < 1e-14


def test_gmres_solves_keep_the_direct_solve_decisions():
    """The library replaces the reference's direct LU by restarted GMRES(40) to a 1e-12
    relative residual.  On a stiff five-field system whose solves restart, the oracle BDF
    with that GMRES (oracle.gmres) takes the same steps as with the direct solve, with
    step sizes and states equal to 1e-8."""
    prob, y0 = five_field_stiff_problem()
    res = {}
    for linear in ("lu", "gmres"):
        with tempfile.TemporaryDirectory() as wd:
            fb = wd + "/o"
            y0.tofile(fb + "ic.dat")
            cfg = orun.RunConfig(n=prob.n, Ns=prob.Ns, Ls=prob.Ls, terms=prob.terms, t1=1.0, dt=0.5, rtol=1e-4,
                                 atol=1e-4, stiff=True, linear=linear)
            summ = orun.run(fb, cfg)
            res[linear] = (summ, np.fromfile(fb + "steps.dat"), np.fromfile(fb + "states.dat"))
    (lu, lu_h, lu_y), (gm, gm_h, gm_y) = res["lu"], res["gmres"]
    assert gm["steps"] == lu["steps"] and gm["attempts"] == lu["attempts"]
    st = gm["linear"]
    assert st["solves"] > 0 and st["cycles"] > st["solves"]
    assert np.max(np.abs(gm_h - lu_h) / np.abs(lu_h)) < 1e-8
    assert rel_err(gm_y, lu_y) < 1e-8
