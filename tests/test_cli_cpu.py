"""The rdcu CLI's front end against the reference binary, without a GPU: the help text
and Y-index table, and the parsed equations printed by -v (both programs print them
before touching the GPU).  The reference binary is built from its sources by
oracle/build_ref.sh; these tests skip when it is absent."""
import os
import subprocess
import tempfile

import pytest

import rdcu_b200 as R
from oracle.problem import cgle_coupling_lines

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "rdcu_ref")
needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")


def run(exe, args, cwd=None):
    return subprocess.run([exe] + args, capture_output=True, text=True, timeout=60, cwd=cwd)


@needs_ref
@pytest.mark.parametrize("args", [["-h"], ["-n", "2", "-N", "4,4", "-h"], ["-h", "-n", "3", "-N", "5,6,7"],
                                  ["-N", "16", "-n", "1"], []])
def test_help_identical(args):
    a, b = run(R.CLI_PATH, args), run(REF, args)
    assert a.returncode == b.returncode == 0
    assert a.stdout == b.stdout


def _equations(out):
    return [l for l in out.splitlines() if "'=" in l]


@needs_ref
@pytest.mark.parametrize("extra", [[], ["-c", "0.5,1,3,2,0,1", "-c", "-1e-1,0,13,1"], ["-c", "2.0,1"]])
def test_verbose_equations_identical(extra):
    with tempfile.TemporaryDirectory() as wd:
        for exe, tag in ((R.CLI_PATH, "a"), (REF, "b")):
            fb = os.path.join(wd, tag)
            open(fb + "coupling.dat", "w").write("\n".join(cgle_coupling_lines(2)) + "\n")
            r = run(exe, ["-v", "-n", "2", "-N", "8,8", "-L", "10,10", "-t", "0"] + extra + [fb])
            if tag == "a":
                mine = _equations(r.stdout)
            else:
                ref = _equations(r.stdout)
        assert mine and mine == ref


def test_filebase_cancels_help():
    with tempfile.TemporaryDirectory() as wd:
        r = run(R.CLI_PATH, ["-h", "-n", "1", "-N", "8", "-t", "0", os.path.join(wd, "x")])
        assert "usage" not in r.stdout
        assert os.path.exists(os.path.join(wd, "x.out"))
