"""Defect lines on the CPU: the oracle against the reference's own outputs (golden
vectors made by tests/golden/make_lines_golden.py from makelines.py), and the host-side
ancestry and driver of rdcu_b200 against the reference's lineids.dat and command lines."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import lines as ol
from tests.helpers import defect_state

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["lines3", "noise", "odd", "thin", "mixed"]
FRAMES = dict(Ns=(24, 20, 28), seed=14, nterms=2, noise=0.3, drift=1.5, count=6)


def golden_components(d, prefix=""):
    e, off = d["edges" + prefix], d["offsets" + prefix]
    return [e[off[c]:off[c + 1]] for c in range(len(off) - 1)]


def same_components(got, ref, Ns, Ls):
    """Same components in the same order, each with the same edges (as unordered cube
    pairs, and bit-identical scaled coordinates)."""
    if len(got) != len(ref):
        return False
    for a, b in zip(got, ref):
        if a.shape != b.shape or not np.array_equal(ol.canonical(a, Ns, Ls), ol.canonical(b, Ns, Ls)):
            return False
        ra = {tuple(sorted(map(tuple, r))) for r in a}
        rb = {tuple(sorted(map(tuple, r))) for r in b}
        if ra != rb:
            return False
    return True


@pytest.mark.parametrize("case", CASES)
def test_oracle_findlines_matches_reference(case):
    d = np.load(os.path.join(GOLD, "lines_%s.npz" % case))
    got = ol.findlines(d["th"], d["Ns"], d["Ls"])
    assert same_components(got, golden_components(d), d["Ns"], d["Ls"])


def frame_phase(k):
    y = defect_state(FRAMES["Ns"], FRAMES["seed"], k, FRAMES["nterms"], FRAMES["noise"], FRAMES["drift"])
    return ol.phase(y, FRAMES["Ns"])


def test_frame_states_are_the_golden_ones():
    d = np.load(os.path.join(GOLD, "lines_frames.npz"))
    for k in range(FRAMES["count"]):
        assert hashlib.sha256(frame_phase(k).tobytes()).hexdigest() == str(d["th_sha256"][k])


def test_oracle_frames_and_correlate_match_reference():
    d = np.load(os.path.join(GOLD, "lines_frames.npz"))
    Ns, Ls = d["Ns"], d["Ls"]
    frames = [golden_components(d, str(k)) for k in range(FRAMES["count"])]
    for k in range(FRAMES["count"]):
        assert same_components(ol.findlines(frame_phase(k), Ns, Ls), frames[k], Ns, Ls), k
    for n in range(1, FRAMES["count"]):
        assert np.array_equal(ol.correlate(frames[n - 1], frames[n], Ns, Ls), d["diffs%d" % n]), n


def test_oracle_correlate_keeps_the_truncation():
    """The later frame's cubes are truncated back from (c * L) / (N - 1): for N = 12,
    L = 7 cube 7 comes back as 6, so a component at x = 7 is at distance 0 from one at 6."""
    Ns, Ls = (12, 12, 12), (7.0, 7.0, 7.0)
    s = lambda c: (np.array(c, dtype=float) * 7.0) / 11.0
    prev = [np.array([[s([6, 0, 0]), s([6, 0, 1])]])]
    cur = [np.array([[s([7, 0, 0]), s([7, 0, 1])]])]
    assert ol.correlate(prev, cur, Ns, Ls)[0, 0] == 0
    assert ol.correlate(cur, prev, Ns, Ls)[0, 0] == 1


def test_ancestry_matches_reference():
    from rdcu_b200.lines import ancestry

    with open(os.path.join(GOLD, "lines_ancestry.json")) as fh:
        g = json.load(fh)
    frames = [[[None] * n for n in f] for f in g["lengths"]]
    ids, cids, edges = ancestry(frames, [np.array(x) for x in g["diffs"]], g["thr"])
    assert [list(map(int, i)) for i in ids] == g["ids"]
    assert [list(map(int, c)) for c in cids] == g["cids"]
    assert [[int(a), int(b)] for a, b in edges] == g["edges"]


def test_ancestry_births_and_splits():
    from rdcu_b200.lines import ancestry

    frames = [[[0] * 5, [0] * 3], [[0] * 4, [0] * 2, [0] * 6]]
    diffs = [np.array([[1, 7], [1, 9], [9, 9]])]  # two children of component 0, one newborn
    ids, cids, edges = ancestry(frames, diffs, 3)
    assert list(ids[1]) == [2, 3, 4] and list(cids[1]) == [0, 2, 3]
    assert edges == [[0, 2], [0, 3]]


def test_driver_commands_and_coupling_match_reference():
    from rdcu_b200.makelines import coupling_lines, parse_args, state_commands

    with open(os.path.join(GOLD, "lines_driver.json")) as fh:
        g = json.load(fh)
    a = parse_args(["--filebase", "FILEBASE"] + g["args"])
    assert [c[1:] for c in state_commands(a, exe="rdcu")] == g["calls"]
    assert coupling_lines(a.b, a.c) == g["coupling"]
