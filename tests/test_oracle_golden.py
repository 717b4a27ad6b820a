"""The oracle pinned against the reference's own outputs (CPU only).

Fixtures under tests/golden were produced by the reference rdcu built from its sources
(oracle/build_ref.sh) and run on a B200 by tests/golden/make_reference_fixtures.py.
The oracle's emulation of the reference driver must reproduce them: initial conditions
bit for bit (glibc rand), RHS and Y blocks to 1e-12, CSR Jacobian pattern exactly and
values to 1e-12, fixed-step trajectories to 1e-10, and identical accepted-step counts
on the short adaptive runs.
"""
import tempfile

import numpy as np
import pytest

from tests.golden.cases import (BDF_SEQ_CASES, CASES, SEQ_CASES, compare_sequence_outputs, fixture, fixture_steps,
                                oracle_run_case, oracle_run_seq)
from tests.helpers import rel_err

RHS_TOL = 1e-12


def _case(name):
    return next(c for c in CASES if c["name"] == name)


@pytest.fixture(scope="module")
def runs():
    cache = {}

    def get(name):
        if name not in cache:
            with tempfile.TemporaryDirectory() as wd:
                cache[name] = oracle_run_case(_case(name), wd)
        return cache[name]

    return get


def _blocks_close(Y, Yref, nblocks, tol):
    Y = Y.reshape(nblocks, -1)
    Yref = Yref.reshape(nblocks, -1)
    for k in range(nblocks):
        scale = max(float(np.max(np.abs(Yref[k]))), 1e-300)
        assert np.max(np.abs(Y[k] - Yref[k])) / scale < tol, k


@pytest.mark.parametrize("name", [c["name"] for c in CASES if c["name"].startswith("spec")])
def test_spectral_rhs_and_blocks(runs, name):
    fx, o = fixture(name), runs(name)
    assert int(fx["returncode"]) == 0
    np.testing.assert_array_equal(o["states"], fx["states"])  # glibc-rand IC, bit for bit
    assert rel_err(o["f"], fx["f"]) < RHS_TOL
    # Y.dat: n*(1+ndim+ndim^2) blocks of N complex values (n = 2 in every case)
    nY = fx["Y"].size // fx["f"].size
    _blocks_close(o["Y"], fx["Y"], nY * 2, RHS_TOL)


@pytest.mark.parametrize("name", [c["name"] for c in CASES if c["name"].startswith("fd")])
def test_fd_rhs_and_jacobian(runs, name):
    fx, o = fixture(name), runs(name)
    np.testing.assert_array_equal(o["states"], fx["states"])
    assert rel_err(o["f"], fx["f"]) < RHS_TOL
    # real FD blocks; the reference leaves the imaginary parts unwritten (zero here)
    assert rel_err(o["Y"].real, fx["Y"].real) < RHS_TOL
    np.testing.assert_array_equal(o["rows"], fx["rows"])
    np.testing.assert_array_equal(o["cols"], fx["cols"])
    assert rel_err(o["vals"], fx["vals"]) < RHS_TOL


def test_fixed_step_trajectory(runs):
    fx, o = fixture("dp45_fixed_2d"), runs("dp45_fixed_2d")
    np.testing.assert_array_equal(o["times"], fx["times"])
    assert o["states"].size == fx["states"].size
    assert rel_err(o["states"], fx["states"]) < 1e-10
    np.testing.assert_array_equal(o["steps"], fx["steps"])


@pytest.mark.parametrize("name", ["dp45_adaptive_2d", "dp45_adaptive_3d", "dp45_adaptive_1d"])
def test_adaptive_step_counts(runs, name):
    fx, o = fixture(name), runs(name)
    assert o["summary"]["steps"] == fixture_steps(fx)
    assert o["steps"].size == fx["steps"].size  # attempts (steps.dat holds h per attempt)
    assert np.max(np.abs(o["steps"] - fx["steps"]) / np.abs(fx["steps"])) < 1e-8
    np.testing.assert_array_equal(o["times"], fx["times"])
    assert rel_err(o["states"], fx["states"]) < 1e-8
    if "f" in fx:
        assert rel_err(o["f"], fx["f"]) < 1e-8


@pytest.mark.parametrize("case", [c for c in SEQ_CASES + BDF_SEQ_CASES if not c.get("out_only")],
                         ids=lambda c: c["name"])
def test_restart_append_and_bdf_sequences(case):
    """-R restarts (fs.dat reload, appended outputs, no initial write), runs that load
    ic.dat (every output appended), and the reference's own BDF path (its sources with a
    solving stand-in for cuDSS), against the reference's files after the last run."""
    fx = fixture(case["name"])
    with tempfile.TemporaryDirectory() as wd:
        o = oracle_run_seq(case, wd)
    nN = fx["states"].size // fx["times"].size
    compare_sequence_outputs(o, fx, nN)
    for i in range(len(case["runs"])):
        assert o["summary_%d" % i]["steps"] == fixture_steps({"out": fx["out_%d" % i]}), i
