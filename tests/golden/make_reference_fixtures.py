"""Runs the golden cases (cases.py) through the reference's own build and stores every
output file as a compressed .npz fixture.

    python tests/golden/make_reference_fixtures.py --ref oracle/_ref/rdcu_ref --ref-lu oracle/_ref/rdcu_ref_lu --out DIR

Needs a GPU (the reference is CUDA-only).  The committed fixtures in tests/golden were
made with this script from the reference sources built by oracle/build_ref.sh.
"""
import argparse
import os
import shlex
import subprocess
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from tests.golden.cases import BDF_SEQ_CASES, CASES, SEQ_CASES, case_ic  # noqa: E402

FILES = {"states": np.float64, "times": np.float64, "steps": np.float64, "f": np.float64,
         "Y": np.complex128, "rows": np.int32, "cols": np.int32, "vals": np.float64, "fs": np.uint8}


def run_case(ref, case, workdir):
    fb = os.path.join(workdir, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    cmd = [ref] + shlex.split(case["args"]) + [fb]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    out = {"argv": np.array(case["args"]), "returncode": np.array(r.returncode),
           "stdout": np.array(r.stdout)}
    for k, dt in FILES.items():
        p = fb + k + ".dat"
        if os.path.exists(p):
            out[k] = np.fromfile(p, dt)
    if os.path.exists(fb + ".out"):
        out["out"] = np.array(open(fb + ".out").read())
    return out


def run_seq_case(ref, case, workdir):
    """The runs of a sequence case in one directory; files after the last run, and each
    run's return code, stdout and .out text."""
    fb = os.path.join(workdir, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    out = {"runs": np.array(case["runs"])}
    for i, args in enumerate(case["runs"]):
        r = subprocess.run([ref] + shlex.split(args) + [fb], capture_output=True, text=True, timeout=600)
        out["returncode_%d" % i] = np.array(r.returncode)
        out["stdout_%d" % i] = np.array(r.stdout)
        if os.path.exists(fb + ".out"):
            out["out_%d" % i] = np.array(open(fb + ".out").read())
    for k, dt in FILES.items():
        p = fb + k + ".dat"
        if os.path.exists(p):
            out[k] = np.fromfile(p, dt)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--ref-lu", default=None, help="the reference built with the solving cuDSS stand-in")
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as wd:
        for case in CASES:
            if a.only and a.only not in case["name"]:
                continue
            res = run_case(a.ref, case, wd)
            np.savez_compressed(os.path.join(a.out, case["name"] + ".npz"), **res)
            print(case["name"], "rc", int(res["returncode"]), sorted(k for k in res if k not in ("argv", "stdout")))
        for case in SEQ_CASES + (BDF_SEQ_CASES if a.ref_lu else []):
            if a.only and a.only not in case["name"]:
                continue
            res = run_seq_case(a.ref_lu if case.get("ref") == "lu" else a.ref, case, wd)
            np.savez_compressed(os.path.join(a.out, case["name"] + ".npz"), **res)
            print(case["name"], sorted(k for k in res if not k.startswith("stdout")))


if __name__ == "__main__":
    main()
