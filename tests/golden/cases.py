"""Golden cases run through the reference's own build (oracle/_ref/rdcu_ref) on a GPU
box by ``make_reference_fixtures.py``; the resulting fixtures pin the oracle (CPU
tests) and the library (GPU tests).  Each case is the reference CLI's argv, its
coupling file and, optionally, an ic.dat made from a seeded numpy generator."""
import numpy as np

from oracle.problem import brusselator_coupling_lines, cgle_coupling_lines

# random dictionary with mixed derivatives, power 0, constant and odd-length terms
# (n = 2, ndim = 3: Y indices 0..25)
MIXED3D = ["0.5,0,0,1", "-0.25,1,10,1,0,1", "0.3,0,14,2", "1.0,1,20,1", "0.7,0,3,1,8,0",
           "-1.2,1,1,3", "0.4,0", "0.9,1,25,1,4,1", "0.2,0,9", "-0.6,0,22,1,1,1"]
MIXED2D = ["1.0,0,0,1", "0.5,0,2,1,1,1", "-0.8,1,4,2", "0.3,1,8,1,0,2", "1.1,0,11,1",
           "-0.4,1,13,1,0,1", "0.6,0,9,1", "0.25,1,5,1,3,1", "-0.5,0,1,3"]
MIXED1D = ["1.0,0,4,1", "-0.7,1,2,1,0,1", "0.5,0,0,3", "0.8,1,5,1", "0.3,0,3,2"]


def _ic(n, N, seed, base=(0.0,), amp=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(base[i % len(base)] + amp * rng.uniform(-1, 1, N))
    return np.concatenate(out)


CASES = [
    # RHS and Y blocks at t = 0 (pseudospectral)
    dict(name="spec2d_cgle_D3", args="-n 2 -N 16,12 -L 20,15 -A 2 -s 1 -t 0 -D3",
         coupling=cgle_coupling_lines(2)),
    dict(name="spec2d_mixed_odd_D3", args="-n 2 -N 9,10 -L 7,5 -A 2 -s 4 -t 0 -D3", coupling=MIXED2D),
    dict(name="spec3d_cgle_D3", args="-n 2 -N 8,6,10 -L 10,12,14 -A 2 -s 2 -t 0 -D3",
         coupling=cgle_coupling_lines(3)),
    dict(name="spec3d_mixed_D3", args="-n 2 -N 6,5,4 -L 3,4,5 -A 1 -s 7 -t 0 -D3", coupling=MIXED3D),
    dict(name="spec1d_mixed_D3", args="-n 2 -N 12 -L 9 -A 2 -s 3 -t 0 -D3", coupling=MIXED1D),
    # fixed-step trajectory (-F, output every step)
    dict(name="dp45_fixed_2d", args="-n 2 -N 32,32 -L 40,40 -A 2 -s 1 -F -t 0.2 -d 0.01 -D1",
         coupling=cgle_coupling_lines(2)),
    # short adaptive runs (accepted-step counts, steps.dat, dense output)
    dict(name="dp45_adaptive_2d", args="-n 2 -N 32,32 -L 40,40 -A 2 -s 1 -t 1 -d 0.25 -D2",
         coupling=cgle_coupling_lines(2)),
    dict(name="dp45_adaptive_3d", args="-n 2 -N 16,16,16 -L 20,20,20 -A 2 -s 2 -t 0.5 -d 0.25 -r 1e-7 -a 1e-7 -D1",
         coupling=cgle_coupling_lines(3)),
    dict(name="dp45_adaptive_1d", args="-n 2 -N 64 -L 50 -A 2 -s 5 -t 2 -d 0.5 -r 1e-6 -a 1e-6 -D1",
         coupling=cgle_coupling_lines(1)),
    # finite differences at t = 0: RHS, real Y blocks and the CSR Jacobian (-S -D4);
    # the reference then stops in bdf_run because cuDSS is absent
    dict(name="fd2d_brusselator_D4", args="-S -n 2 -N 8,8 -L 16,16 -t 0 -D4",
         coupling=brusselator_coupling_lines(), ic=dict(n=2, N=64, seed=3, base=(1.0, 3.0), amp=0.1)),
    dict(name="fd2d_cgle_D4", args="-S -n 2 -N 10,8 -L 12,10 -A 2 -s 1 -t 0 -D4",
         coupling=cgle_coupling_lines(2)),
    dict(name="fd3d_mixed_D4", args="-S -n 2 -N 5,4,6 -L 3,4,5 -A 1 -s 7 -t 0 -D4", coupling=MIXED3D),
    dict(name="fd1d_mixed_D4", args="-S -n 2 -N 12 -L 9 -A 2 -s 3 -t 0 -D4", coupling=MIXED1D),
]


# Runs in sequence in one directory: -R restarts from FILEBASEfs.dat (rdcu.cu:944-990)
# and append-mode outputs whenever an IC was loaded (rdcu.cu:1013-1016).  The
# fixtures hold every output file after the last run and each run's .out text.
_C2 = "-n 2 -N 32,32 -L 40,40 -A 2 -s 1"
SEQ_CASES = [
    # DP45 to t = 0.5, then -R to t = 1: the restart appends states/times/steps and
    # rewrites fs.dat; no initial state is written on reload
    dict(name="restart_dp45_2d", coupling=cgle_coupling_lines(2),
         runs=[_C2 + " -t 0.5 -d 0.25 -D1", _C2 + " -t 1 -d 0.25 -D1 -R"]),
    # fixed steps, restarted
    dict(name="restart_fixed_2d", coupling=cgle_coupling_lines(2),
         runs=[_C2 + " -F -t 0.05 -d 0.01 -D1", _C2 + " -F -t 0.1 -d 0.01 -D1 -R"]),
    # a DP45 fs.dat reloaded by a stiff run: "Couldn't read order!" (rdcu.cu:968-975);
    # the reference's BDF then stops at its cuDSS set-up, so only the .out lines up to
    # the restart message are compared
    dict(name="restart_dp45_to_bdf_2d", coupling=cgle_coupling_lines(2),
         runs=[_C2 + " -t 0.5 -d 0.25 -D1", "-S " + _C2 + " -t 1 -d 0.25 -D1 -R"], out_only=True),
    # ic.dat present: both runs start from it and append every output
    dict(name="append_ic_2d", coupling=cgle_coupling_lines(2),
         runs=["-n 2 -N 16,16 -L 20,20 -t 0.5 -d 0.25 -D2", "-n 2 -N 16,16 -L 20,20 -t 0.5 -d 0.25 -D2"],
         ic=dict(n=2, N=256, seed=9, amp=1.0)),
]


# The reference's BDF path (bdf.cu) run by oracle/_ref/rdcu_ref_lu: the unmodified
# reference sources with a solving stand-in for cuDSS (oracle/cudss_stub/cudss_lu.cpp,
# cuSOLVER's host sparse LU).  "ref": "lu" marks the cases that need it.
_B2 = "-S -n 2 -N 32,32 -L 40,40 -A 2 -s 1"
BDF_SEQ_CASES = [
    # a stiff run of the 2D CGLE (finite differences, variable-order BDF)
    dict(name="bdf_cgle_2d", coupling=cgle_coupling_lines(2), runs=[_B2 + " -t 2 -d 0.5 -D1"], ref="lu"),
    # the Brusselator from an ic.dat (offsets (1, 3) plus noise)
    dict(name="bdf_brusselator_2d", coupling=brusselator_coupling_lines(),
         runs=["-S -n 2 -N 32,32 -L 16,16 -t 3 -d 1 -D1"], ic=dict(n=2, N=1024, seed=3, base=(1.0, 3.0), amp=0.1),
         ref="lu"),
    # BDF to t = 1, then -R to t = 2: fs.dat carries the order and the D blocks
    # (rdcu.cu:322-339, reloaded at :977-983)
    dict(name="restart_bdf_2d", coupling=cgle_coupling_lines(2),
         runs=[_B2 + " -t 1 -d 0.5 -D1", _B2 + " -t 2 -d 0.5 -D1 -R"], ref="lu"),
    # a DP45 fs.dat reloaded by a stiff run ("Couldn't read order!"), the whole run
    dict(name="restart_dp45_to_bdf_lu_2d", coupling=cgle_coupling_lines(2),
         runs=[_C2 + " -t 0.5 -d 0.25 -D1", "-S " + _C2 + " -t 1 -d 0.25 -D1 -R"], ref="lu"),
]


def case_ic(case):
    spec = case.get("ic")
    if not spec:
        return None
    return _ic(spec["n"], spec["N"], spec["seed"], spec.get("base", (0.0,)), spec.get("amp", 1.0))


def oracle_run_case(case, workdir):
    """Runs one case through the oracle's emulation of the reference driver and returns
    the output files as arrays (same keys as the fixtures)."""
    import os
    import shlex

    from oracle import run as orun
    from oracle.problem import parse_term

    fb = os.path.join(workdir, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    cfg, _, _, _ = orun.config_from_argv(shlex.split(case["args"]) + [fb])
    cfg.terms = cfg.terms + [parse_term(s) for s in case["coupling"]]
    summary = orun.run(fb, cfg)
    out = {"summary": summary}
    kinds = {"states": np.float64, "times": np.float64, "steps": np.float64, "f": np.float64,
             "Y": np.complex128, "rows": np.int32, "cols": np.int32, "vals": np.float64, "fs": np.uint8}
    for k, dt in kinds.items():
        p = fb + k + ".dat"
        if os.path.exists(p):
            out[k] = np.fromfile(p, dt)
    return out


def oracle_run_seq(case, workdir):
    """The runs of a sequence case through the oracle's driver emulation, in one
    directory; returns the output files after the last run."""
    import os
    import shlex

    from oracle import run as orun
    from oracle.problem import parse_term

    fb = os.path.join(workdir, case["name"])
    with open(fb + "coupling.dat", "w") as fh:
        fh.write("\n".join(case["coupling"]) + "\n")
    ic = case_ic(case)
    if ic is not None:
        ic.tofile(fb + "ic.dat")
    out = {}
    for i, args in enumerate(case["runs"]):
        cfg, _, _, _ = orun.config_from_argv(shlex.split(args) + [fb])
        cfg.terms = cfg.terms + [parse_term(s) for s in case["coupling"]]
        out["summary_%d" % i] = orun.run(fb, cfg)
    kinds = {"states": np.float64, "times": np.float64, "steps": np.float64, "f": np.float64, "fs": np.uint8}
    for k, dt in kinds.items():
        p = fb + k + ".dat"
        if os.path.exists(p):
            out[k] = np.fromfile(p, dt)
    return out


def fixture(name):
    import os

    return dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), name + ".npz")))


def fixture_steps(fx):
    """Accepted-step count from the reference's .out ("steps: N")."""
    for line in str(fx["out"]).splitlines():
        if line.startswith("steps:"):
            return int(line.split()[1])
    return None


def fs_parts(raw, nN):
    """fs.dat as written by the reference (rdcu.cu:322-339): y (nN doubles), t, h, and
    for stiff runs the int32 order and order*nN doubles D_1..D_order."""
    raw = np.asarray(raw, np.uint8)
    out = {"y": raw[: 8 * nN].view(np.float64), "th": raw[8 * nN: 8 * nN + 16].view(np.float64)}
    rest = raw[8 * nN + 16:]
    if rest.size >= 4:
        out["order"] = int(rest[:4].view(np.int32)[0])
        out["D"] = rest[4:].view(np.float64)
    return out


def compare_sequence_outputs(o, fx, nN, states_tol=1e-8):
    """Every output file of a sequence case against the reference's fixture: times
    exactly, states and step sizes to states_tol, f.dat to 1e-7, fs.dat's state, t, h,
    order and D blocks."""
    def rel(a, b):
        return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)

    np.testing.assert_array_equal(o["times"], fx["times"])
    assert o["states"].size == fx["states"].size
    assert rel(o["states"], fx["states"]) < states_tol
    assert o["steps"].size == fx["steps"].size
    assert np.max(np.abs(o["steps"] - fx["steps"]) / np.abs(fx["steps"])) < states_tol
    if "f" in fx:
        assert rel(o["f"], fx["f"]) < 1e-7
    a, b = fs_parts(o["fs"], nN), fs_parts(fx["fs"], nN)
    assert rel(a["y"], b["y"]) < states_tol
    assert np.max(np.abs(a["th"] - b["th"]) / np.abs(b["th"])) < 1e-10
    assert ("order" in a) == ("order" in b)
    if "order" in b:
        assert a["order"] == b["order"]
        assert a["D"].size == b["D"].size
        assert rel(a["D"], b["D"]) < 1e3 * states_tol  # differences: D_k of h^k scale
