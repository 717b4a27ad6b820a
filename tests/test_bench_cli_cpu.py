"""The CLI workloads of bench.py on CPU: the rate comes from the .out progress lines
(N x difference of cumulative steps / difference of elapsed seconds between the first and
last output), as for the reference; a stand-in executable writes a known .out."""
import stat

import bench


def _fake_cli(tmp_path, lines, rc=0):
    """A stand-in CLI: copies a prepared .out to FILEBASE.out (FILEBASE is its last
    argument) and writes a 4 KB states.dat."""
    src = tmp_path / "prepared.out"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "fake_rdcu"
    exe.write_text('#!/bin/sh\nfb="$(eval echo \\${$#})"\ncp "%s" "${fb}.out"\n'
                   'head -c 4096 /dev/zero > "${fb}states.dat"\nexit %d\n' % (src, rc))
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    return str(exe)


def test_rate_from_progress_lines(tmp_path):
    out = ["Using random initial conditions", "0.010\t1.000e+00\t9.900e+01\t0.010000\t10\t",
           "0.500\t3.000e+00\t3.000e+00\t0.020000\t110\t", "1.000\t5.000e+00\t0.000e+00\t0.020000\t210\t",
           "", "steps: 210", "runtime: 5.500000"]
    exe = _fake_cli(tmp_path, out)
    wl = dict(cli="-n 2 -N 16,16 -t 1", Ns=(16, 16), outputs=3)
    res, err = bench.cli_run(exe, wl)
    assert err is None
    assert res["value"] == 256 * 200 / 4.0
    assert res["steps"] == 210 and res["window_steps"] == 200 and res["outputs"] == 3
    assert res["runtime_s"] == 5.5 and res["states_bytes"] == 4096


def test_failed_run_is_reported(tmp_path):
    exe = _fake_cli(tmp_path, ["rdcu initialization failed: x"], rc=1)
    res, err = bench.cli_run(exe, dict(cli="-n 2", Ns=(8, 8), outputs=2))
    assert res is None and "rc 1" in err


def test_launches_per_attempt_separate_and_fused():
    """Per-attempt launch counts of the profiled passes: five forward and inverse x
    passes without fusion; with the fused row pass (stages 2-5) stage 2's forward pass,
    four fused launches, stage 6's inverse pass and stage 7's two x passes.  Either way
    the 3D attempt's spectral passes run six times each, and the fused attempt is the 27
    launches (with the controller) of its launch list."""
    sep = ["fwd_x", "c2c_axis1_fwd", "mid_axis0", "c2c_axis1_inv", "inv_x_dictionary", "fwd_x_stage7", "inv_x_stage7"]
    w = [bench.launches_per_attempt_of(p, sep) for p in sep]
    assert w == [5, 6, 6, 6, 5, 1, 1]
    assert sum(w) + 1 == 31
    fused = sep + ["inv_fwd_row", "fwd_x_stage2"]
    w = dict((p, bench.launches_per_attempt_of(p, fused)) for p in fused)
    assert w == {"fwd_x": 0, "c2c_axis1_fwd": 6, "mid_axis0": 6, "c2c_axis1_inv": 6, "inv_x_dictionary": 1,
                 "fwd_x_stage7": 1, "inv_x_stage7": 1, "inv_fwd_row": 4, "fwd_x_stage2": 1}
    assert sum(w.values()) + 1 == 27
