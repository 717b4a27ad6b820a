"""GPU parity of the defect-line path (rdcu_lines_*): line cubes, components, edges and
the frame-to-frame distance matrix against the reference's golden vectors and the
oracle.  Integer and index results are compared exactly; the scaled coordinates are
compared bit for bit."""
import os

import numpy as np
import pytest

from oracle import lines as ol
from tests.helpers import defect_state
from tests.test_lines_cpu import CASES, FRAMES, GOLD, frame_phase, golden_components, same_components

pytestmark = pytest.mark.gpu


def _lines(Ns, Ls):
    from rdcu_b200.lines import Lines

    return Lines(Ns, Ls)


@pytest.mark.parametrize("case", CASES)
def test_findlines_matches_reference_golden(cuda, case):
    from rdcu_b200 import lines as L

    d = np.load(os.path.join(GOLD, "lines_%s.npz" % case))
    got = L.findlines(d["th"], d["Ns"], d["Ls"])
    assert same_components(got, golden_components(d), d["Ns"], d["Ls"])


def test_edges_are_canonical_and_cubes_grouped(cuda):
    d = np.load(os.path.join(GOLD, "lines_mixed.npz"))
    h = _lines(d["Ns"], d["Ls"])
    n, ne, nc = h.find(d["th"], 1)
    for comp in h.lines():  # (u, v), u < v, ascending
        q = np.round(comp * (d["Ns"] - 1) / d["Ls"]).astype(np.int64)
        idx = np.ravel_multi_index(q.reshape(-1, 3).T, tuple(d["Ns"])).reshape(-1, 2)
        assert np.array_equal(idx, ol.canonical(comp, d["Ns"], d["Ls"]))
    idx, off = h.cubes()
    cubes = np.nonzero(ol.line_cubes(d["th"]).ravel())[0]
    comp, _, _ = ol.components(cubes, d["Ns"])
    assert n == cubes.size and nc == comp.max() + 1 and off[-1] == n
    for c in range(nc):
        assert np.array_equal(idx[off[c]:off[c + 1]], cubes[comp == c])
    h.close()


@pytest.mark.parametrize("Ns,seed,nterms,noise", [((32, 24, 40), 21, 3, 0.1), ((16, 16, 16), 22, 0, 2.5),
                                                  ((2, 30, 17), 23, 2, 0.5), ((45, 2, 33), 24, 1, 0.2),
                                                  ((64, 64, 64), 25, 4, 0.05)])
def test_state_input_matches_oracle(cuda, Ns, seed, nterms, noise):
    """State input (phase formed on the GPU) and phase input, host and device sources."""
    Ls = tuple(0.4 * n + 1.0 for n in Ns)
    y = defect_state(Ns, seed, 0, nterms, noise)
    th = ol.phase(y, Ns)
    ref = ol.findlines(th, Ns, Ls)
    h = _lines(Ns, Ls)
    h.find(y, 0)
    assert same_components(h.lines(), ref, Ns, Ls)
    yd = cuda.tensor(y, dtype=cuda.float64, device="cuda")
    cuda.cuda.synchronize()
    h.find(yd, 0)
    assert same_components(h.lines(), ref, Ns, Ls)
    h.find(cuda.tensor(th.ravel(), dtype=cuda.float64, device="cuda"), 1)
    assert same_components(h.lines(), ref, Ns, Ls)
    h.close()


def test_thousands_of_components(cuda):
    """Isolated points of phase pi on a spaced lattice: one small component each (4096 of
    them: two 8-bit passes of the component sort)."""
    Ns, Ls = (64, 64, 64), (10.0, 20.0, 30.0)
    th = np.zeros(Ns)
    th[1::4, 2::4, 3::4] = np.pi
    ref = ol.findlines(th, Ns, Ls)
    assert len(ref) == 4096
    h = _lines(Ns, Ls)
    h.find(th, 1)
    assert same_components(h.lines(), ref, Ns, Ls)
    h.close()


def test_empty_frame(cuda):
    Ns, Ls = (8, 9, 10), (1.0, 2.0, 3.0)
    h = _lines(Ns, Ls)
    assert h.find(np.full(Ns, 0.5), 1) == (0, 0, 0)
    assert h.lines() == []
    idx, off = h.cubes()
    assert idx.size == 0 and list(off) == [0]
    g = _lines(Ns, Ls)
    th = np.zeros(Ns)
    th[3, 3, 3] = np.pi
    g.find(th, 1)
    assert h.correlate(g).shape == (0, 1) and g.correlate(h).shape == (1, 0)
    h.close()
    g.close()


def test_correlate_device_frames_match_reference(cuda):
    d = np.load(os.path.join(GOLD, "lines_frames.npz"))
    Ns, Ls = d["Ns"], d["Ls"]
    hs = [_lines(Ns, Ls), _lines(Ns, Ls)]
    for k in range(FRAMES["count"]):
        cur = hs[k % 2]
        cur.find(frame_phase(k), 1)
        assert same_components(cur.lines(), golden_components(d, str(k)), Ns, Ls), k
        if k:
            assert np.array_equal(cur.correlate(hs[(k - 1) % 2]), d["diffs%d" % k]), k
    for h in hs:
        h.close()


def test_correlate_mirror_matches_reference(cuda):
    from rdcu_b200 import lines as L

    d = np.load(os.path.join(GOLD, "lines_frames.npz"))
    Ns, Ls = d["Ns"], d["Ls"]
    frames = [golden_components(d, str(k)) for k in range(FRAMES["count"])]
    for n in range(1, FRAMES["count"]):
        assert np.array_equal(L.correlate(n, frames, Ns, Ls, 1024, "cuda"), d["diffs%d" % n]), n


def test_correlate_large_frames_against_oracle(cuda):
    Ns, Ls = (48, 40, 56), (30.0, 25.0, 35.0)
    a = _lines(Ns, Ls)
    b = _lines(Ns, Ls)
    a.find(defect_state(Ns, 31, 0, 3, 0.2, 1.5), 0)
    b.find(defect_state(Ns, 31, 1, 3, 0.2, 1.5), 0)
    ref = ol.correlate(a.lines(), b.lines(), Ns, Ls)
    assert ref.size > 4
    assert np.array_equal(b.correlate(a), ref)
    a.close()
    b.close()


def test_savelines_reads_states_file(cuda, tmp_path):
    from rdcu_b200 import lines as L

    Ns, Ls = (20, 18, 16), (9.0, 8.0, 7.0)
    frames = [defect_state(Ns, 41, k, 2, 0.1) for k in range(3)]
    fn = str(tmp_path / "xstates.dat")
    np.concatenate(frames).tofile(fn)
    got = L.savelines(1, fn, np.array(Ns), np.array(Ls), 1)
    assert same_components(got, ol.findlines(ol.phase(frames[2], Ns), Ns, Ls), Ns, Ls)
    faces = L.loadfaces(0, str(tmp_path / "x"), Ns, 2)
    assert np.array_equal(faces[3], frames[2].reshape((2,) + Ns)[:, -1, :, :])


def test_errors(cuda):
    import rdcu_b200 as R
    from rdcu_b200.lines import Lines, findlines

    with pytest.raises(R.RdcuError) as e:
        Lines((1, 8, 8), (1.0, 1.0, 1.0))
    assert e.value.code == R.RDCU_ERR_INVALID
    h = Lines((8, 8, 8), (1.0, 1.0, 1.0))
    with pytest.raises(R.RdcuError) as e:
        h.edges()
    assert e.value.code == R.RDCU_ERR_STATE
    with pytest.raises(R.RdcuError) as e:
        h.correlate_sets([np.array([0, 600])], [np.array([1])])
    assert e.value.code == R.RDCU_ERR_INVALID
    with pytest.raises(ValueError):
        findlines(np.zeros((8, 8, 8)), (8, 8, 8), (1.0, 1.0, 1.0), device="cpu")
    h.close()


def test_driver_end_to_end(cuda, tmp_path):
    """python -m rdcu_b200.makelines on a small grid: the rdcu CLI writes the frames, the
    driver's lines/diffs/lineids files equal the oracle on those frames."""
    import pickle

    from rdcu_b200 import makelines as M
    from rdcu_b200.lines import ancestry, read_frame

    fb = str(tmp_path / "x")
    args = ["--filebase", fb, "--Ns", "16", "12", "20", "--Ls", "10", "8", "12", "--T0", "0.01", "--dt0", "0.001",
            "--T1", "0.2", "--dt1", "0.1", "--T", "1.0", "--dt", "0.2", "--seed", "3"]
    assert M.main(args) == 0
    a = M.parse_args(args)
    Ns, Ls = np.array(a.Ns), np.array(a.Ls)
    n0 = 1 + int(a.T0 / a.dt0) + int(a.T1 / a.dt1)
    nt = int((a.T - a.T1) / a.dt)
    load = lambda k: pickle.load(open(fb + k + ".dat", "rb"))
    lines, diffs, (ids, cids, edges), faces = load("lines"), load("diffs"), load("lineids"), load("faces")
    assert len(lines) == nt == len(faces) and len(diffs) == nt - 1
    for n in range(nt):
        ref = ol.findlines(ol.phase(read_frame(fb + "states.dat", Ns, n0 + n), Ns), Ns, Ls)
        assert len(ref) > 0 and same_components(lines[n], ref, Ns, Ls), n
    for n in range(1, nt):
        assert np.array_equal(diffs[n - 1], ol.correlate(lines[n - 1], lines[n], Ns, Ls)), n
    i2, c2, e2 = ancestry(lines, diffs, a.thr)
    assert all(np.array_equal(x, y) for x, y in zip(ids, i2)) and edges == e2


def test_profile_passes(cuda):
    """rdcu_lines_profile times the pass groups of one find and leaves that frame's results."""
    Ns, Ls = (32, 24, 40), (20.0, 15.0, 25.0)
    y = defect_state(Ns, 21, 0, 3, 0.1)
    h = _lines(Ns, Ls)
    p = h.profile(y, 0, reps=3)
    assert [x[0] for x in p] == ["phase", "faces", "mark", "compact", "components", "sort", "edges"]
    assert all(ms > 0 for _, ms, _ in p) and p[1][2] == 9.0 * np.prod(Ns)
    assert same_components(h.lines(), ol.findlines(ol.phase(y, Ns), Ns, Ls), Ns, Ls)
    assert [x[0] for x in h.profile(ol.phase(y, Ns), 1, reps=2)][0] == "faces"
    h.close()


def test_prefetched_frames(cuda):
    """A two-handle sequence with each next frame staged by rdcu_lines_prefetch while the
    current one is found gives the same lines and distance matrices as direct finds."""
    import rdcu_b200 as R

    Ns, Ls = (32, 24, 40), (20.0, 15.0, 25.0)
    frames = [cuda.tensor(defect_state(Ns, 41, k, 3, 0.1, 1.0)).pin_memory() for k in range(5)]
    ref = _lines(Ns, Ls)
    want_lines = []
    for k in range(5):
        ref.find(frames[k].numpy(), 0)
        want_lines.append(ref.lines())
    hs = [_lines(Ns, Ls), _lines(Ns, Ls)]
    hs[0].find(frames[0], 0)
    hs[1].prefetch(frames[1], 0)
    for k in range(1, 5):
        c, p = hs[k % 2], hs[(k - 1) % 2]
        if k + 1 < 5:
            p.prefetch(frames[k + 1], 0)
        c.find(None, 0)
        assert same_components(c.lines(), want_lines[k], Ns, Ls), k
        assert np.array_equal(c.correlate(p), ol.correlate(want_lines[k - 1], want_lines[k], Ns, Ls)), k
    with pytest.raises(R.RdcuError) as e:
        hs[0].find(None, 0)  # nothing staged
    assert e.value.code == R.RDCU_ERR_STATE
    hs[0].prefetch(frames[0], 0)
    with pytest.raises(R.RdcuError) as e:
        hs[0].find(None, 1)  # staged frame is a state, not a phase field
    assert e.value.code == R.RDCU_ERR_STATE
    hs[0].find(frames[2], 0)  # an explicit frame after a pending prefetch
    assert same_components(hs[0].lines(), want_lines[2], Ns, Ls)
    for h in hs + [ref]:
        h.close()
