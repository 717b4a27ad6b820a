"""Runs a few DP45 attempts of a CGLE problem and times every pass kernel of one fused
RHS stage (rdcu_profile_passes); prints one JSON line.  Intended as a small, fixed
workload for profilers such as Nsight Compute:

    python -m tests.profile_case 256,256,128 [--attempts 3] [--reps 2]
"""
import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from rdcu_b200 import Solver, random_ic  # noqa: E402
from rdcu_b200.problems import cgle_coupling_lines  # noqa: E402


def cgle_terms(ndim, b=2.0, c=0.8):
    out = []
    for s in cgle_coupling_lines(ndim, b, c):
        t = s.split(",")
        out.append((float(t[0]), [int(x) for x in t[1:]]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("grid", help="comma-separated grid sizes, e.g. 256,256,128")
    ap.add_argument("--length", type=float, default=200.0)
    ap.add_argument("--attempts", type=int, default=3)
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args()
    Ns = tuple(int(x) for x in a.grid.split(","))
    s = Solver(2, Ns, (a.length,) * len(Ns), cgle_terms(len(Ns)))
    N = int(np.prod(Ns))
    y = random_ic(2, N, 2.0, 0.0, 2)
    s.set_state(0.0, 1e-3, y.ctypes.data)
    acc = s.advance(a.attempts)
    passes = s.profile_passes(reps=a.reps)
    print(json.dumps({"grid": Ns, "accepted": acc, "passes": [
        {"name": p[0], "ms": p[1], "bytes": p[2], "GBps": p[2] / (p[1] / 1e3) / 1e9} for p in passes]}))
    s.close()


if __name__ == "__main__":
    main()
