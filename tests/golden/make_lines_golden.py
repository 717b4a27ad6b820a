"""Golden vectors for the defect-line path, produced by the reference's own Python
(makelines.py: findlines_np, correlate_np, and its __main__ driver and ancestry block).

    python tests/golden/make_lines_golden.py --reference "$RDCU_REFERENCE_DIR" --out tests/golden

Needs the reference sources (and networkx, as the reference does); runs on the CPU.
Writes lines_<case>.npz (the phase field and the per-component edges), lines_frames.npz
(a frame sequence -- states from tests.helpers.defect_state with FRAMES' parameters,
their phases' sha256 -- with the reference's edges and correlate matrices),
lines_ancestry.json (the reference's lineids.dat for that sequence) and lines_driver.json
(the coupling file and rdcu command lines its driver writes for one set of flags).
"""
import argparse
import hashlib
import json
import os
import pickle
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from tests.helpers import defect_state  # noqa: E402

# name: (Ns, Ls, seed, nterms, noise); white-noise states use nterms 0 and a large noise
CASES = {
    "lines3": ((12, 10, 14), (5.0, 6.0, 7.0), 1, 3, 0.05),
    "noise": ((8, 10, 12), (5.0, 6.0, 7.0), 2, 0, 3.0),
    "odd": ((9, 7, 5), (3.0, 2.0, 4.0), 3, 2, 0.3),
    "thin": ((2, 6, 5), (1.0, 2.0, 3.0), 4, 1, 1.0),
    "mixed": ((24, 20, 16), (50.0, 30.0, 20.0), 5, 4, 0.2),
}
FRAMES = dict(Ns=(24, 20, 28), Ls=(7.0, 30.0, 37.5), seed=14, nterms=2, noise=0.3, drift=1.5, count=6)


def _pack(lines):
    off = np.cumsum([0] + [len(l) for l in lines])
    edges = np.concatenate(lines, axis=0) if lines else np.zeros((0, 2, 3))
    return edges, off


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("RDCU_REFERENCE_DIR"), required="RDCU_REFERENCE_DIR" not in os.environ)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    import makelines as ml

    for name, (Ns, Ls, seed, nterms, noise) in CASES.items():
        y = defect_state(Ns, seed, 0, nterms, noise)
        ys = y.reshape((2,) + Ns)
        th = np.atan2(ys[1], ys[0]) + np.pi
        lines = ml.findlines_np(th, np.array(Ns), np.array(Ls), 64)
        edges, off = _pack(lines)
        np.savez_compressed(os.path.join(a.out, "lines_%s.npz" % name), th=th, Ns=np.array(Ns),
                            Ls=np.array(Ls), edges=edges, offsets=off)
        print(name, "components", len(lines), "edges", int(off[-1]))

    F = FRAMES
    frames, sums = [], []
    for k in range(F["count"]):
        y = defect_state(F["Ns"], F["seed"], k, F["nterms"], F["noise"], F["drift"])
        ys = y.reshape((2,) + F["Ns"])
        th = np.atan2(ys[1], ys[0]) + np.pi
        frames.append(ml.findlines_np(th, np.array(F["Ns"]), np.array(F["Ls"]), 64))
        sums.append(hashlib.sha256(th.tobytes()).hexdigest())
    diffs = [ml.correlate_np(n, frames, np.array(F["Ns"]), np.array(F["Ls"]), 64) for n in range(1, F["count"])]
    packed = [_pack(l) for l in frames]
    np.savez_compressed(os.path.join(a.out, "lines_frames.npz"), th_sha256=np.array(sums), Ns=np.array(F["Ns"]),
                        Ls=np.array(F["Ls"]), **{"edges%d" % k: p[0] for k, p in enumerate(packed)},
                        **{"offsets%d" % k: p[1] for k, p in enumerate(packed)},
                        **{"diffs%d" % (n + 1): d for n, d in enumerate(diffs)})
    print("frames components", [len(l) for l in frames])

    # the reference's ancestry (its __main__ block), fed the same lines and diffs
    with tempfile.TemporaryDirectory() as wd:
        fb = os.path.join(wd, "x")
        for nm, obj in (("lines", frames), ("faces", []), ("diffs", diffs)):
            with open(fb + nm + ".dat", "wb") as fh:
                pickle.dump(obj, fh)
        thr = 3
        cmd = [sys.executable, os.path.join(a.reference, "makelines.py"), "--filebase", fb, "--states", "0",
               "--T", str(F["count"]), "--T1", "0", "--dt", "1", "--thr", str(thr),
               "--Ns"] + [str(n) for n in F["Ns"]] + ["--Ls"] + [str(l) for l in F["Ls"]]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise SystemExit(r.stderr)
        with open(fb + "lineids.dat", "rb") as fh:
            ids, cids, edges = pickle.load(fh)
    out = dict(thr=thr, lengths=[[len(c) for c in f] for f in frames], diffs=[d.tolist() for d in diffs],
               ids=[np.asarray(i).tolist() for i in ids], cids=[np.asarray(c).tolist() for c in cids],
               edges=[[int(x) for x in e] for e in edges])
    with open(os.path.join(a.out, "lines_ancestry.json"), "w") as fh:
        json.dump(out, fh)
    print("ancestry ids", out["ids"], "edges", out["edges"])

    # the driver's coupling file and rdcu command lines: makelines.py run with a stand-in
    # ./rdcu that records its arguments
    with tempfile.TemporaryDirectory() as wd:
        fake = os.path.join(wd, "rdcu")
        with open(fake, "w") as fh:
            fh.write('#!/bin/sh\necho "$@" >> "%s"\n' % os.path.join(wd, "calls.txt"))
        os.chmod(fake, 0o755)
        fb = os.path.join(wd, "x")
        args = ["--filebase", fb, "--lines", "0", "--states", "1", "--Ns", "16", "12", "8", "--Ls", "7.5", "6",
                "5.25", "--b", "0.7", "--c", "-1.3", "--seed", "5", "--T0", "0.01", "--dt0", "0.001", "--T", "0.5",
                "--dt", "0.1", "--T1", "0.3", "--dt1", "0.05"]
        r = subprocess.run([sys.executable, os.path.join(a.reference, "makelines.py")] + args, cwd=wd,
                           capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise SystemExit(r.stderr)
        calls = [l.replace(fb, "FILEBASE").split() for l in open(os.path.join(wd, "calls.txt")).read().splitlines()]
        coupling = open(fb + "coupling.dat").read().splitlines()
    with open(os.path.join(a.out, "lines_driver.json"), "w") as fh:
        json.dump({"args": args[2:], "calls": calls, "coupling": coupling}, fh, indent=0)
    print("driver calls", calls)


if __name__ == "__main__":
    main()
