"""3D CGLE defect-line tracking: the reference's makelines.py driver on librdcu.

    python -m rdcu_b200.makelines --filebase DIR/x [--Ns 128 128 128] [--Ls 50 50 50] ...

Same flags, same files as the reference (makelines.py:191-387):

1. ``--states 1``: writes FILEBASE``coupling.dat`` (the 22-term CGLE with --b, --c) and
   runs the rdcu CLI three times -- a fixed-step burn-in to T0, then adaptive output
   every dt1 from T0 to T1 and every dt to T -- so that FILEBASE``states.dat`` holds
   the frames (makelines.py:247-268).  The CLI is this package's ``bin/rdcu``.
2. ``--lines 1``: ``lines.dat`` (per frame, per component, the edges as (E, 2, 3)
   arrays), ``faces.dat`` (six boundary faces per frame), ``diffs.dat`` (correlate
   matrices of consecutive frames) and ``lineids.dat`` (ids, colour ids and ancestry
   edges), each a pickle like the reference's.

The per-frame work runs on the GPU through two ``rdcu_b200.lines.Lines`` handles: each
frame is found in one handle and correlated against the previous frame still on the
device in the other, instead of the reference's process pool over frames.  Existing
lines.dat / faces.dat / diffs.dat files are loaded instead of recomputed, as the
reference does.
"""
from __future__ import annotations

import argparse
import os
import pickle
import subprocess
import sys
import timeit

import numpy as np

from . import CLI_PATH
from .lines import STATE, Lines, _device_index, ancestry, correlate, loadfaces, read_frame


def coupling_lines(b: float, c: float) -> list:
    """The 3D CGLE coupling the reference writes (makelines.py:249-254), '%f'-formatted."""
    return ['1.0,0,0,1', '1.0,0,8,1', '1.0,0,16,1', '1.0,0,24,1', '-%f,0,9,1' % b, '-%f,0,17,1' % b,
            '-%f,0,25,1' % b, '-1.0,0,0,3', '-1.0,0,0,1,1,2', '1.0,1,1,1', '1.0,1,9,1', '1.0,1,17,1', '1.0,1,25,1',
            '%f,1,8,1' % b, '%f,1,16,1' % b, '%f,1,24,1' % b, '-1.0,1,0,2,1,1', '-1.0,1,1,3', '%f,1,0,3' % c,
            '%f,1,0,1,1,2' % c, '-%f,0,0,2,1,1' % c, '-%f,0,1,3' % c]


def state_commands(a, exe: str = CLI_PATH) -> list:
    """The three rdcu runs of makelines.py:260-268 (argument lists)."""
    common = ["-N", "%i,%i,%i" % tuple(a.Ns), "-L", "%f,%f,%f" % tuple(a.Ls), "-s", str(a.seed), "-n", "2", "-D1"]
    return [
        [exe, "-s", "1", "-t", "%f" % a.T0, "-d", "%f" % a.dt0] + common + ["-F", a.filebase],
        [exe, "-s", "1", "-t", "%f" % a.T1, "-d", "%f,%f,0,%f" % (a.dt1, a.dt0, a.dt)] + common + ["-R", a.filebase],
        [exe, "-s", "1", "-t", "%f" % a.T, "-d", "%f" % a.dt] + common + ["-R", a.filebase],
    ]


def parse_args(argv=None):
    p = argparse.ArgumentParser(description="3DCGLE defect lines.")
    p.add_argument("--filebase", type=str, required=True, dest="filebase", help="Base string for file output")
    p.add_argument("--Ns", type=int, nargs=3, default=[128, 128, 128], dest="Ns", help="Grid points in each dimension")
    p.add_argument("--Ls", type=float, nargs=3, default=[50.0, 50.0, 50.0], dest="Ls", help="Domain lengths")
    p.add_argument("--b", type=float, default=0.5, dest="b", help="CGLE b parameter")
    p.add_argument("--c", type=float, default=2.0, dest="c", help="CGLE c parameter")
    p.add_argument("--seed", type=int, default=100, dest="seed", help="Random seed")
    p.add_argument("--T0", type=float, default=0.1, dest="T0", help="Fixed step burn in time")
    p.add_argument("--dt0", type=float, default=1e-3, dest="dt0", help="Fixed step burn in time step")
    p.add_argument("--T", type=float, default=1000, dest="T", help="Total integration time")
    p.add_argument("--dt", type=float, default=10.0, dest="dt", help="Final output time step")
    p.add_argument("--T1", type=float, default=900, dest="T1", help="Time to start tracking lines")
    p.add_argument("--dt1", type=float, default=0.1, dest="dt1", help="Initial output time step")
    p.add_argument("--lines", type=int, default=1, dest="dolines", help="Flag to track lines")
    p.add_argument("--states", type=int, default=1, dest="dostates", help="Flag to generate states")
    p.add_argument("--threads", type=int, default=16, dest="threads", help="Accepted for compatibility (unused)")
    p.add_argument("--chunk", type=int, default=1024, dest="chunk", help="Accepted for compatibility (unused)")
    p.add_argument("--rm", type=int, default=0, dest="rm", help="Remove states")
    p.add_argument("--thr", type=int, default=5, dest="thr", help="Threshold distance for correlate")
    p.add_argument("--device", type=str, default="cuda", dest="device", help="CUDA device (cuda or cuda:k)")
    return p.parse_args(argv)


def _load_or(path, make):
    if os.path.exists(path):
        with open(path, "rb") as fh:
            return pickle.load(fh)
    obj = make()
    with open(path, "wb") as fh:
        pickle.dump(obj, fh)
    return obj


def track(a) -> tuple:
    """lines.dat, faces.dat, diffs.dat and lineids.dat for the frames in states.dat."""
    Ns, Ls = np.array(a.Ns), np.array(a.Ls)
    n0 = 1 + int(a.T0 / a.dt0) + int(a.T1 / a.dt1)
    nt = int((a.T - a.T1) / a.dt)
    states = a.filebase + "states.dat"
    dev = _device_index(a.device)
    computed = {}

    def run_frames():
        hs = [Lines(Ns, Ls, dev), Lines(Ns, Ls, dev)]
        lines, diffs = [], []
        for n in range(nt):
            cur = hs[n % 2]
            cur.find(read_frame(states, Ns, n0 + n), STATE)
            lines.append([np.array(c) for c in cur.lines()])
            if n:
                diffs.append(cur.correlate(hs[(n - 1) % 2]))
        for h in hs:
            h.close()
        computed["diffs"] = diffs
        return lines

    start = timeit.default_timer()
    lines = _load_or(a.filebase + "lines.dat", run_frames)
    print("lines time: ", timeit.default_timer() - start, flush=True)
    start = timeit.default_timer()
    faces = _load_or(a.filebase + "faces.dat", lambda: [loadfaces(n, a.filebase, Ns, n0) for n in range(nt)])
    print("faces load time: ", timeit.default_timer() - start, flush=True)
    if a.rm and os.path.exists(states):
        os.remove(states)

    def run_diffs():
        if "diffs" in computed:
            return computed["diffs"]
        return [correlate(n, lines, Ns, Ls, a.chunk, a.device) for n in range(1, nt)]

    start = timeit.default_timer()
    results = _load_or(a.filebase + "diffs.dat", run_diffs)
    print("correlate time: ", timeit.default_timer() - start, flush=True)
    start = timeit.default_timer()
    ids, cids, edges = ancestry(lines, results, a.thr)
    with open(a.filebase + "lineids.dat", "wb") as fh:
        pickle.dump((ids, cids, edges), fh)
    print("line ancestry time: ", timeit.default_timer() - start, flush=True)
    return lines, faces, results, (ids, cids, edges)


def main(argv=None) -> int:
    a = parse_args(argv)
    print(*(sys.argv if argv is None else ["makelines"] + list(argv)))
    if a.dostates:
        with open("%scoupling.dat" % a.filebase, "w") as fh:
            for line in coupling_lines(a.b, a.c):
                print(line, file=fh)
        for cmd in state_commands(a):
            print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=False)
    if a.dolines:
        track(a)
    return 0


if __name__ == "__main__":
    sys.exit(main())
