"""GPU: the rdcu CLI of this library against the reference's own outputs.

Each golden case runs through rdcu_b200/bin/rdcu with the reference's argv and
coupling file; every output file is compared with the fixture the reference build
wrote (same tolerances as the oracle pin: RHS/Y 1e-12, Jacobian pattern exact and
values 1e-12, fixed-step trajectories 1e-10, identical accepted-step counts).
"""
import os
import shlex
import subprocess
import tempfile

import numpy as np
import pytest

from tests.golden.cases import BDF_SEQ_CASES, CASES, SEQ_CASES, case_ic, compare_sequence_outputs, fixture, fixture_steps
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rdcu_b200", "bin", "rdcu")
KINDS = {"states": np.float64, "times": np.float64, "steps": np.float64, "f": np.float64,
         "Y": np.complex128, "rows": np.int32, "cols": np.int32, "vals": np.float64}


def run_cli(case, wd):
    fb = os.path.join(wd, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    r = subprocess.run([CLI] + shlex.split(case["args"]) + [fb], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {k: np.fromfile(fb + k + ".dat", dt) for k, dt in KINDS.items() if os.path.exists(fb + k + ".dat")}
    out["out"] = open(fb + ".out").read()
    return out


def _steps(text):
    for line in text.splitlines():
        if line.startswith("steps:"):
            return int(line.split()[1])


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_cli_matches_reference(case):
    fx = fixture(case["name"])
    with tempfile.TemporaryDirectory() as wd:
        o = run_cli(case, wd)
    for k in KINDS:
        assert (k in o) == (k in fx), k
    np.testing.assert_array_equal(o["states"][: fx["states"].size // max(1, fx["times"].size)],
                                  fx["states"][: fx["states"].size // max(1, fx["times"].size)])
    np.testing.assert_array_equal(o["times"], fx["times"])
    name = case["name"]
    if name.startswith("spec") or name.startswith("fd"):
        assert rel_err(o["f"], fx["f"]) < 1e-12
        nY = fx["Y"].size // fx["f"].size
        Y, Yr = o["Y"].reshape(nY * 2, -1), fx["Y"].reshape(nY * 2, -1)
        for k in range(nY * 2):
            if name.startswith("fd"):
                assert rel_err(Y[k].real, Yr[k].real) < 1e-12, k
            else:
                sc = max(np.max(np.abs(Yr[k])), 1e-300)
                assert np.max(np.abs(Y[k] - Yr[k])) / sc < 1e-12, k
    if name.startswith("fd"):
        np.testing.assert_array_equal(o["rows"], fx["rows"])
        np.testing.assert_array_equal(o["cols"], fx["cols"])
        assert rel_err(o["vals"], fx["vals"]) < 1e-12
    if name == "dp45_fixed_2d":
        assert rel_err(o["states"], fx["states"]) < 1e-10
        np.testing.assert_array_equal(o["steps"], fx["steps"])
    if name.startswith("dp45_adaptive"):
        assert _steps(o["out"]) == fixture_steps(fx)
        assert o["steps"].size == fx["steps"].size
        assert np.max(np.abs(o["steps"] - fx["steps"]) / np.abs(fx["steps"])) < 1e-8
        assert rel_err(o["states"], fx["states"]) < 1e-8


def run_seq_cli(case, wd):
    fb = os.path.join(wd, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    out = {}
    for i, args in enumerate(case["runs"]):
        r = subprocess.run([CLI] + shlex.split(args) + [fb], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        out["out_%d" % i] = open(fb + ".out").read()
    for k, dt in list(KINDS.items()) + [("fs", np.uint8)]:
        if os.path.exists(fb + k + ".dat"):
            out[k] = np.fromfile(fb + k + ".dat", dt)
    return out


def message_lines(text):
    """The .out lines after the argv line: status messages as they are, progress lines as
    (fraction of the run, h, accepted steps) -- their elapsed-time columns differ -- and
    no runtime line."""
    res = []
    for line in str(text).splitlines()[1:]:
        if not line.strip() or line.startswith("runtime:"):
            continue
        if line[0].isdigit():
            c = line.split("\t")
            res.append((c[0], c[3], c[4]))
        else:
            res.append(line)
    return res


@pytest.mark.parametrize("case", SEQ_CASES + BDF_SEQ_CASES, ids=[c["name"] for c in SEQ_CASES + BDF_SEQ_CASES])
def test_cli_sequence_matches_reference(case):
    """-R restarts, ic.dat append runs and BDF runs: each run's .out messages, and every
    output file after the last run, against the reference's."""
    fx = fixture(case["name"])
    with tempfile.TemporaryDirectory() as wd:
        o = run_seq_cli(case, wd)
    for i in range(len(case["runs"])):
        ours, ref = message_lines(o["out_%d" % i]), message_lines(fx["out_%d" % i])
        if case.get("out_only") and i == len(case["runs"]) - 1:
            # the reference's BDF stops at its cuDSS set-up: messages up to the restart
            k = next(j for j, l in enumerate(ref) if isinstance(l, str) and l.startswith("Restarting at"))
            assert ours[: k + 1] == ref[: k + 1], (ours[: k + 1], ref[: k + 1])
        else:
            assert ours == ref, (i, ours, ref)
    if case.get("out_only"):
        return
    compare_sequence_outputs(o, fx, fx["states"].size // fx["times"].size)
