"""GPU parity: DP45 stepping of librdcu against the oracle's restatement of dp45.cu.

* fixed steps (-F): trajectories within 1e-10 relative (max-norm);
* adaptive steps: identical accept/reject sequence and step sizes within 1e-9 relative
  over short horizons (the CGLE is chaotic; short horizons keep rounding differences
  from growing);
* dense output, FSAL and the whole-integration event stream (rdcu_solve).
"""
import numpy as np
import pytest

from oracle import dp45 as odp
from oracle import spectral as osp
from oracle.problem import Problem, cgle_terms
from tests.helpers import rel_err, smooth_field, spec_terms

pytestmark = pytest.mark.gpu


def _setup(torch, prob, y0, **kw):
    import rdcu_b200 as R

    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), **kw)
    yd = torch.tensor(y0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    return s, yd


def _oracle(prob, y0, fixed, rtol=1e-8, atol=1e-8):
    st = odp.DP45(y0, atol, rtol, fixed, lambda t, y: osp.rhs(y, prob))
    st.k[0] = st.dydt(0.0, st.y)
    return st


def test_fixed_step_trajectory(cuda):
    rng = np.random.default_rng(11)
    prob = Problem(2, (32, 32), (40.0, 40.0), cgle_terms(2))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    s, yd = _setup(cuda, prob, y0, fixed=True)
    h = 1e-2
    s.set_state(0.0, h, yd.data_ptr())
    o = _oracle(prob, y0, True)
    t = to = 0.0
    for _ in range(20):
        acc, t, h2 = s.step(t, h)
        ok, to, _ = o.step(to, h, 0.0, np.inf)
        o.k[0] = o.k[6]
        assert acc and ok
    out = cuda.empty_like(yd)
    tt, hh, _ = s.get_state(out.data_ptr())
    assert abs(tt - to) < 1e-14
    assert rel_err(out.cpu().numpy(), o.y) < 1e-10


@pytest.mark.parametrize("Ns,Ls,rtol", [((32, 32), (40.0, 40.0), 1e-8), ((64,), (30.0,), 1e-6),
                                        ((8, 8, 16), (12.0, 12.0, 20.0), 1e-7),
                                        ((256, 4, 8), (200.0, 4.0, 8.0), 1e-8),
                                        ((128, 8, 6), (100.0, 6.0, 5.0), 1e-8),
                                        ((8, 128, 128), (6.0, 100.0, 100.0), 1e-8)])
def test_adaptive_sequence(cuda, Ns, Ls, rtol):
    rng = np.random.default_rng(len(Ns))
    prob = Problem(2, Ns, Ls, cgle_terms(len(Ns)))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    s, yd = _setup(cuda, prob, y0, rtol=rtol, atol=rtol)
    h = 1e-2
    s.set_state(0.0, h, yd.data_ptr())
    o = _oracle(prob, y0, False, rtol, rtol)
    t = to = 0.0
    hg = ho = h
    for i in range(25):
        acc, t, hg = s.step(t, hg)
        ok, to, ho = o.step(to, ho, 0.0, np.inf)
        if ok:
            o.k[0] = o.k[6]
        assert acc == ok, i
        assert abs(hg - ho) <= 1e-9 * abs(ho), (i, hg, ho)
        assert abs(t - to) <= 1e-12 * max(1.0, abs(to))
    out = cuda.empty_like(yd)
    s.get_state(out.data_ptr())
    assert rel_err(out.cpu().numpy(), o.y) < 1e-9


def test_plane_passes_dp45_3d(cuda, monkeypatch):
    """3D CGLE 128^3 with RDCU_PLANE_PASSES=1 (x rows and axis-1 lines of 128 points:
    the x passes that also transform along axis 1, one cluster per plane): ten adaptive
    attempts against the default axis-1 passes on TMA tiles -- the same accept/reject
    sequence, step sizes and states within 1e-9 (the axis-1 transforms round
    differently; the error norm's cancellation amplifies that) -- and the passes
    profiled are the plane passes, stage 7 with its error epilogue included."""
    rng = np.random.default_rng(5)
    prob = Problem(2, (128, 128, 128), (200.0, 200.0, 200.0), cgle_terms(3))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    runs = []
    for plane in (True, False):
        if plane:
            monkeypatch.setenv("RDCU_PLANE_PASSES", "1")
        else:
            monkeypatch.delenv("RDCU_PLANE_PASSES", raising=False)
        s, yd = _setup(cuda, prob, y0)
        s.set_state(0.0, 1e-3, yd.data_ptr())
        names = [p[0] for p in s.profile_passes(reps=1)]
        assert ("fwd_plane" in names and "inv_plane_stage7" in names) == plane, names
        s.set_state(0.0, 1e-3, yd.data_ptr())
        t, h, seq = 0.0, 1e-3, []
        for _ in range(10):
            acc, t, h = s.step(t, h)
            seq.append((acc, t, h))
        out = cuda.empty_like(yd)
        s.get_state(out.data_ptr())
        runs.append((seq, out.cpu().numpy()))
        s.close()
    (sa, ya), (sb, yb) = runs
    for i, ((a1, t1, h1), (a2, t2, h2)) in enumerate(zip(sa, sb)):
        assert a1 == a2, i
        assert abs(h1 - h2) <= 1e-9 * abs(h2) and abs(t1 - t2) <= 1e-9 * max(1.0, abs(t2)), (i, h1, h2)
    assert rel_err(ya, yb) < 1e-9


@pytest.mark.parametrize("Ns,Ls", [((6, 10, 256), (5.0, 8.0, 200.0)), ((128, 128, 128), (200.0, 200.0, 200.0))])
def test_fused_row_passes_dp45_3d(cuda, monkeypatch, Ns, Ls):
    """3D CGLE with 256- and 128-point x rows: by default a stage's inverse x pass and
    the next stage's forward x pass run as one kernel (k_inv_fwd_row, stages 2..5);
    RDCU_FUSED_ROWS=0 runs them as separate kernels.  Ten adaptive attempts each: the
    same accept/reject sequence, step sizes and states within 1e-9 (the fused forward
    transform packs the two fields of a row into one complex line where k_fwd_x packs
    two rows of a field, so the spectra round differently), the fused passes are the
    ones profiled, and on the small grid the fused run follows the oracle's attempts."""
    rng = np.random.default_rng(9)
    prob = Problem(2, Ns, Ls, cgle_terms(3))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    runs = []
    for fused in (True, False):
        if fused:
            monkeypatch.delenv("RDCU_FUSED_ROWS", raising=False)
        else:
            monkeypatch.setenv("RDCU_FUSED_ROWS", "0")
        s, yd = _setup(cuda, prob, y0)
        s.set_state(0.0, 1e-3, yd.data_ptr())
        names = [p[0] for p in s.profile_passes(reps=1)]
        assert ("inv_fwd_row" in names and "fwd_x_stage2" in names) == fused, names
        s.set_state(0.0, 1e-3, yd.data_ptr())
        t, h, seq = 0.0, 1e-3, []
        for _ in range(10):
            acc, t, h = s.step(t, h)
            seq.append((acc, t, h))
        out = cuda.empty_like(yd)
        s.get_state(out.data_ptr())
        runs.append((seq, out.cpu().numpy()))
        s.close()
    (sa, ya), (sb, yb) = runs
    for i, ((a1, t1, h1), (a2, t2, h2)) in enumerate(zip(sa, sb)):
        assert a1 == a2, i
        assert abs(h1 - h2) <= 1e-9 * abs(h2) and abs(t1 - t2) <= 1e-9 * max(1.0, abs(t2)), (i, h1, h2)
    assert rel_err(ya, yb) < 1e-9
    if prob.N <= 20000:
        o = _oracle(prob, y0, False)
        to, ho = 0.0, 1e-3
        for i, (acc, t, h) in enumerate(sa):
            ok, to, ho = o.step(to, ho, 0.0, np.inf)
            if ok:
                o.k[0] = o.k[6]
            assert acc == ok, i
            assert abs(h - ho) <= 1e-9 * abs(ho), (i, h, ho)
        assert rel_err(ya, o.y) < 1e-9


def test_dense_output(cuda):
    rng = np.random.default_rng(21)
    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.3)
    s, yd = _setup(cuda, prob, y0)
    h = 0.02
    s.set_state(0.0, h, yd.data_ptr())
    o = _oracle(prob, y0, False)
    t = to = 0.0
    ho = h
    for _ in range(10):  # until an accepted step (same decisions in both)
        tl = t
        acc, t, h = s.step(t, h)
        ok, to, ho = o.step(to, ho, 0.0, np.inf)
        assert acc == ok
        if acc:
            break
    assert acc
    ye = cuda.empty_like(yd)
    for frac in (0.0, 0.3, 0.77, 1.0):
        te = tl + (t - tl) * frac
        s.eval(te, ye.data_ptr())
        assert rel_err(ye.cpu().numpy(), o.eval(to, te)) < 1e-10


def test_solve_events_match_oracle_run(cuda):
    """rdcu_solve's event stream against the reference driver loop (dp45_run + step_eval)."""
    rng = np.random.default_rng(31)
    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y0 = rng.uniform(-1, 1, 2 * prob.N)
    s, yd = _setup(cuda, prob, y0, rtol=1e-6, atol=1e-6)
    s.set_state(0.0, 0.01, yd.data_ptr())
    t_eval = [0.1, 0.2, 0.3]
    ev = {"h": [], "acc": [], "evals": [], "ckpt": []}

    def cb(e):
        if e.kind == 0:
            ev["h"].append(e.h)
            ev["acc"].append(e.accepted)
        elif e.kind == 1:
            ev["evals"].append((e.t_eval, s.copy_to_numpy(e.y, 2 * prob.N)))
        else:
            ev["ckpt"].append((e.t, e.h))
        return 0

    s.solve(0.3, t_eval, callback=cb)
    o = odp.DP45(y0, 1e-6, 1e-6, False, lambda t, y: osp.rhs(y, prob))
    oh, oacc, oev = [], [], []
    ei = [0]

    def se(t, h, y, ok):
        oh.append(h)
        oacc.append(ok)
        if ok:
            while ei[0] < len(t_eval) and t >= t_eval[ei[0]]:
                oev.append((t_eval[ei[0]], o.eval(t, t_eval[ei[0]])))
                ei[0] += 1

    o.run(0.0, 0.01, 0.0, np.inf, 0.3, se)
    assert ev["acc"] == [int(a) for a in oacc]
    assert np.max(np.abs(np.array(ev["h"]) - np.array(oh)) / np.abs(oh)) < 1e-9
    assert len(ev["evals"]) == len(oev) == 3
    for (te, yg), (teo, yo) in zip(ev["evals"], oev):
        assert te == teo
        assert rel_err(yg, yo) < 1e-9
    assert len(ev["ckpt"]) == 3
    acc, att = s.counters()
    assert acc == sum(oacc) and att == len(oacc)


def test_advance_beyond_the_attempt_log(cuda):
    """rdcu_advance re-arms the device controller past its 4096-entry attempt log."""
    rng = np.random.default_rng(21)
    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y0 = smooth_field(rng, prob, amp=0.5)
    s, yd = _setup(cuda, prob, y0, fixed=True)
    s.set_state(0.0, 1e-4, yd.data_ptr())
    assert s.advance(5000) == 5000
    t, h, _ = s.get_state()
    assert abs(t - 0.5) < 1e-12 and h == 1e-4
    s.close()
