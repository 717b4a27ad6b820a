"""Benchmark: grid-pt.steps/s of DP45 pseudospectral integration on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Workload (default "cgle3d_256"): 3D complex Ginzburg-Landau as two FP64 fields on a
256^3 periodic grid, L = 200^3, the 22-term coupling of the reference's 3D example
(b = 2, c = 0.8), uniform random [-1, 1] initial condition from glibc rand() with seed 2,
adaptive DP45 at rtol = atol = 1e-8 (the reference CLI
run ``-n 2 -N 256,256,256 -L 200,200,200 -A 2 -s 2 -t T -d T,0.001``; the first step
is 1e-3 because the reference cannot start from its default dt/100, see WORKLOADS).  Synthetic data: there
is no dataset; the IC is the reference's own generator.

A bench step is TAU units of simulation time of that trajectory.  W warm-up steps
integrate [0, W*TAU] untimed (the white-noise transient), then K steps [W*TAU,
(W+K)*TAU] are timed; the metric counts accepted DP45 steps (rejected attempts are
overhead), value = grid points x accepted steps / seconds.  Inputs are far larger than
the 126 MB L2 (every stage moves ~0.27 GB arrays), so no L2 flush is needed.

* ``value``: device-resident integration (rdcu_solve, controller on the device), timed
  with CUDA events on the library's stream.
* ``e2e``: the same window through the public C ABI with host buffers: rdcu_set_state
  from a pinned host array, rdcu_solve with one output at the window's end copied to the
  host, rdcu_get_state to the host; wall clock around the calls.
* ``roofline``: the dominant pass kernel (most device time per attempt: per-launch time
  from rdcu_profile_passes times its launches per attempt), achieved = bytes the pass
  must move per launch / its CUDA-event time.
* ``cpu_baseline``: the oracle's numpy/scipy restatement (scipy.fft, all host cores) on
  one DP45 attempt of the same workload from the warm state.
* ``--impl reference``: the reference's own nvcc sm_100a build (cuFFT/cuBLAS; the
  reference has no CPU path).  Its clock starts at program start, so set-up must stay out
  of the window: 3D runs twice, to W*TAU and to (W+K)*TAU (grids up to 2M points: a
  window ten times as long), value = grid points x (difference of accepted steps) /
  (difference of runtimes); 2D runs once with outputs every W*TAU and takes the rate
  between the progress lines at W*TAU and at the end.

Multi-GPU (torchrun, N > 1): replicas.  The problem does not shard; every rank
integrates its own copy, timing is the max over ranks, value is the sum of all ranks'
grid-pt.steps over that time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shlex
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt·steps/s"
TAU = 0.05  # simulation time per bench step

# h0: first step.  The reference's own default (dt/100 = 0.2 for dt = 20) overflows on
# the white-noise start and its never-rewritten imaginary half of Y block 0 then keeps
# the NaN in every later transform, so no step is ever accepted; both arms start at 1e-3.
WORKLOADS = {
    "cgle3d_256": dict(Ns=(256, 256, 256), Ls=(200.0, 200.0, 200.0), seed=2, h0=1e-3),
    "cgle3d_128": dict(Ns=(128, 128, 128), Ls=(200.0, 200.0, 200.0), seed=2, h0=1e-3),
    "cgle2d_256": dict(Ns=(256, 256), Ls=(100.0, 100.0), seed=1, h0=1e-3),
    "cgle2d_128": dict(Ns=(128, 128), Ls=(100.0, 100.0), seed=1, h0=1e-3),
    # 512 independent 2D CGLE problems of uneven size, stepped as one ensemble (see run_ensemble)
    "ensemble_cgle2d_512": dict(members=512, sizes=(64, 96, 128, 192, 256), seed=3, h0=1e-3, tau=0.1),
    # stiff path: 2D Brusselator, 5-point finite differences, variable-order BDF (see run_bdf)
    "bdf_brusselator_256": dict(Ns=(256, 256), Ls=(64.0, 64.0), seed=3, h0=1e-3, tau=1.0),
    # discrete adjoint: gradient of a terminal mismatch over 5000 fixed steps (see run_adjoint)
    "adjoint_cgle2d_256": dict(Ns=(256, 256), Ls=(200.0, 200.0), seed=1, h=1e-3, T=5.0, K=50),
    # whole CLI runs with outputs, same flags for both CLIs (see run_cli): C1 as given, and
    # C2's output-every-time-unit run shortened to T = 4 (5 frames of 268 MB)
    "cli_c1_cgle2d_128": dict(cli="-n 2 -N 128,128 -L 100,100 -A 2 -s 1 -t 100 -d 1 -r 1e-8 -a 1e-8 -D1",
                              Ns=(128, 128), outputs=101),
    "cli_c2_cgle3d_256_d1": dict(cli="-n 2 -N 256,256,256 -L 200,200,200 -A 2 -s 2 -t 4 -D1", Ns=(256, 256, 256),
                                 outputs=5),
    # defect lines of 3D CGLE frames at the line tracker's default grid (see run_lines)
    "lines_cgle3d_128": dict(Ns=(128, 128, 128), Ls=(50.0, 50.0, 50.0), seed=7, terms=8, noise=0.1, drift=0.7,
                             frames_per_step=16, ring=48),
}


def cgle_lines(ndim):
    from rdcu_b200.problems import cgle_coupling_lines  # the coupling text the reference notebook writes

    return cgle_coupling_lines(ndim)


def parse_terms(lines):
    out = []
    for s in lines:
        toks = [t for t in s.split(",") if t]
        out.append((float(toks[0]), [int(t) for t in toks[1:]]))
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.skip = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the first sample can take a while to appear: start timing once it has
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.skip = len(self.lines)  # taken before the timed region
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        during = self.lines[self.skip:] or self.lines  # a short region may see no sample of its own
        for l in during:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- our arm
# DRAM bytes (read + write) per launch of each pass of DP45 stages 4 and 7 on the 3D
# CGLE, from one ncu capture per kernel (`ncu --set full ... python -m tests.profile_case
# 256,256,128 --attempts 2 --reps 1`, 8.39 M grid points; the axis-1 inverse pass is
# the forward one's kernel on the same bytes); traffic grows with the grid points, so
# the full-size workload's figure is this one scaled by its points.  inv_fwd_row (the
# fused stage 4 -> 5 pass) and the axis-1 passes are captures of the current kernels;
# the stage-7 entries predate the forward pass writing only the slope sums (its capture
# includes the scale array, 134 MB at this size, which it no longer writes).
NCU_POINTS = 256 * 256 * 128
# DRAM bytes per launch of the defect-line grid passes on the 128^3 workload frames, from
# one ncu capture (`ncu --set full -k regex:"k_(faces|hook|corr)" ... bench.py --workload
# lines_cgle3d_128 --steps 1 --warmup 3`): k_faces reads the 16.8 MB phase field once.
NCU_TRAFFIC_LINES = {"faces": 16.8e6}
NCU_TRAFFIC_3D = {"fwd_x": 772.4e6, "c2c_axis1_fwd": 218.8e6, "mid_axis0": 225.0e6, "c2c_axis1_inv": 218.8e6,
                  "inv_x_dictionary": 373.6e6, "fwd_x_stage7": 1296.7e6, "inv_x_stage7": 656.5e6,
                  "inv_fwd_row": 1171.4e6}


def combine_ranks(seconds, work, device):
    """Whole-job figures of N replicas: the slowest rank's time and the sum of all ranks'
    work (every rank calls this; one all-reduce each)."""
    import torch
    import torch.distributed as dist

    mx = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[0])


def run_ours(args, rank, world, local_rank):
    import torch

    import rdcu_b200 as R

    wl = WORKLOADS[args.workload]
    Ns, Ls = wl["Ns"], wl["Ls"]
    N = int(np.prod(Ns))
    nN = 2 * N
    torch.cuda.set_device(local_rank)
    terms = parse_terms(cgle_lines(len(Ns)))
    s = R.Solver(2, Ns, Ls, terms, rtol=1e-8, atol=1e-8, device=local_rank)
    y0 = R.random_ic(2, N, 2.0, 0.0, wl["seed"])
    h0 = wl["h0"]
    T_A, T_B = args.warmup * TAU, (args.warmup + args.steps) * TAU
    s.set_state(0.0, h0, y0.ctypes.data)
    # warm-up: integrate the transient [0, T_A] (device loop)
    s.solve(T_A, [])
    yA = np.empty(nN)
    tA, hA, _ = s.get_state(yA.ctypes.data)
    stream = torch.cuda.ExternalStream(s.stream, device=local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    # timed: [T_A, T_B] on the device
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        s.solve(T_B, [])
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    acc, att = s.counters()
    tB, hB, _ = s.get_state()
    if dist:
        dist.barrier()
        ms_max, work = combine_ranks(ms, float(acc) * N, "cuda")
    else:
        ms_max, work = ms, float(acc) * N
    value = work / (ms_max / 1e3)

    # per-pass roofline of one fused RHS stage (device, CUDA events)
    passes = s.profile_passes(reps=10)
    peak, peak_kind = load_peaks()
    # the dominant pass is the one with the most device time per attempt
    weights = [launches_per_attempt_of(p[0], [q[0] for q in passes]) for p in passes]
    top = max(zip(passes, weights), key=lambda pw: pw[0][1] * pw[1])[0]
    achieved = top[2] / (top[1] / 1e3) / 1e9
    total_ms = sum(p[1] * w for p, w in zip(passes, weights))
    # whole-step view: algorithmic bytes of one DP45 step (1040 N bytes for the 3D CGLE:
    # 41 state-sized arrays + one spectral round trip per field per direction, 6 stages)
    b_step = (1040.0 if len(Ns) == 3 else 656.0) * N
    step_ms = ms / max(1, att)

    # e2e through the public API with host buffers, same window from the saved state
    s2 = s  # set_state resets the handle
    pin = torch.empty(nN, dtype=torch.float64).pin_memory()
    pin.numpy()[:] = yA
    out_pin = torch.empty(nN, dtype=torch.float64).pin_memory()
    last = torch.empty(nN, dtype=torch.float64).pin_memory()
    if dist:
        dist.barrier()

    def cb(ev):
        if ev.kind == R.EV_EVAL:
            s2.memcpy(out_pin.data_ptr(), ev.y, nN * 8)
        return 0

    w0 = time.perf_counter()
    s2.set_state(tA, hA, pin.data_ptr())
    s2.solve(T_B, [T_B], callback=cb)
    s2.get_state(last.data_ptr())
    e2e_s = time.perf_counter() - w0
    acc2, att2 = s2.counters()
    if dist:
        e2e_s, e2e_work = combine_ranks(e2e_s, float(acc2) * N, "cuda")
    else:
        e2e_work = float(acc2) * N
    e2e_value = e2e_work / e2e_s

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(Ns, Ls, yA, tA, hA)
    s.close()
    line = {
        "metric": METRIC, "value": value, "unit": "grid-pt·steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(Ns), "L": list(Ls), "fields": 2,
                   "dictionary": "CGLE b=2 c=0.8 (%d terms)" % len(terms), "method": "DP45 pseudospectral",
                   "rtol": 1e-8, "atol": 1e-8, "ic": "glibc rand seed %d, [-1,1]" % wl["seed"],
                   "window_sim_time": [T_A, T_B], "tau_per_step": TAU,
                   "accepted_steps": acc, "attempts": att, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs > L2 (no flush needed)"},
        # the passes of six stages and the controller, per attempt
        "gpu_launches": (sum(weights) + 1) * att * world,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": nN * 8 / args.steps,
                "d2h_bytes_per_step": 2 * nN * 8 / args.steps, "accepted_steps": acc2, "seconds": e2e_s},
        "roofline": {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (NCU_TRAFFIC_3D[top[0]] * N / NCU_POINTS)
                     if len(Ns) == 3 and top[0] in NCU_TRAFFIC_3D else None,
                     "traffic_note": "ncu DRAM bytes of the 256x256x128 capture scaled by grid points"
                                     if len(Ns) == 3 else "no capture for 1D/2D",
                     "algorithmic_bytes_per_launch": top[2], "launch_ms": top[1],
                     "passes": [{"name": p[0], "ms": p[1], "GBps": p[2] / (p[1] / 1e3) / 1e9,
                                 "launches_per_attempt": w, "share": p[1] * w / total_ms}
                                for p, w in zip(passes, weights)],
                     "step": {"algorithmic_bytes": b_step, "ms_per_attempt": step_ms,
                              "achieved_GBps": b_step / (step_ms / 1e3) / 1e9,
                              "frac": b_step / (step_ms / 1e3) / 1e9 / peak}},
    }
    if cpu:
        line["cpu_baseline"] = cpu
    return line


def run_adjoint(args):
    """Gradient workload: 2D CGLE 256^2, L = 200, fixed h = 1e-3 to T = 5 (5000 steps),
    checkpoints every 50 steps.  Loss = mean squared mismatch at T against a target the
    method generates from coefficients scaled by 1 + 0.05 N(0,1) (numpy seed 7); gradients
    with respect to all 18 coefficients and the 2 x 256^2 initial state.  value = grid
    points x steps / (forward with checkpoints + backward) seconds; cost_ratio = that time
    over a plain forward run (rdcu_advance) of the same steps; fd_check = central
    differences with eps = 1e-6 along 8 random unit coefficient directions."""
    import torch

    import rdcu_b200 as R

    wl = WORKLOADS[args.workload]
    Ns, Ls = wl["Ns"], wl["Ls"]
    N = int(np.prod(Ns))
    nN = 2 * N
    nsteps = int(round(wl["T"] / wl["h"]))
    hs = [wl["h"]] * nsteps
    terms = parse_terms(cgle_lines(2))
    C = np.array([c for c, _ in terms])
    s = R.Solver(2, Ns, Ls, terms, fixed=True)
    stream = torch.cuda.ExternalStream(s.stream)
    y0 = torch.tensor(R.random_ic(2, N, 2.0, 0.0, wl["seed"]), dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(7)
    Cp = C * (1.0 + 0.05 * rng.normal(size=C.size))
    target = torch.empty_like(y0)
    yT = torch.empty_like(y0)
    g = torch.empty_like(y0)
    torch.cuda.synchronize()
    s.set_coefficients(list(Cp))
    s.adjoint_forward(y0.data_ptr(), hs, wl["K"], target.data_ptr())
    s.set_coefficients(list(C))

    def loss(out):
        return float(((out - target) ** 2).mean())

    # warm-up (graph capture of the segment sweeps happens here)
    s.adjoint_forward(y0.data_ptr(), hs[:2 * wl["K"]], wl["K"], yT.data_ptr())
    lam = (2.0 / nN) * (yT - target)
    s.adjoint_backward(lam.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    with ClockSampler(0) as clk:
        s.set_state(0.0, wl["h"], y0.data_ptr())
        _, t_plain = timed(lambda: s.advance(nsteps))
        _, t_fwd = timed(lambda: s.adjoint_forward(y0.data_ptr(), hs, wl["K"], yT.data_ptr()))
        L0 = loss(yT)
        lam = (2.0 / nN) * (yT - target)
        torch.cuda.synchronize()
        gC, t_bwd = timed(lambda: s.adjoint_backward(lam.data_ptr(), g.data_ptr()))
    gC = np.array(gC)
    # e2e: host arrays through the C ABI (the library stages them)
    y0_h = torch.empty(nN, dtype=torch.float64).pin_memory()
    y0_h.copy_(y0.cpu())
    yT_h = torch.empty(nN, dtype=torch.float64).pin_memory()
    g_h = torch.empty(nN, dtype=torch.float64).pin_memory()
    tgt_h = target.cpu().numpy()
    w0 = time.perf_counter()
    s.adjoint_forward(y0_h.data_ptr(), hs, wl["K"], yT_h.data_ptr())
    lam_h = torch.from_numpy((2.0 / nN) * (yT_h.numpy() - tgt_h)).pin_memory()
    s.adjoint_backward(lam_h.data_ptr(), g_h.data_ptr())
    e2e_s = time.perf_counter() - w0
    # central differences along random unit coefficient directions
    fd = []
    for _ in range(8):
        d = rng.normal(size=C.size)
        d /= np.linalg.norm(d)
        eps = 1e-6
        vals = []
        for sgn in (1, -1):
            s.set_coefficients(list(C + sgn * eps * d))
            s.adjoint_forward(y0.data_ptr(), hs, nsteps, yT.data_ptr())
            vals.append(loss(yT))
        fdv = (vals[0] - vals[1]) / (2 * eps)
        adj = float(np.dot(gC, d))
        fd.append({"fd": fdv, "adjoint": adj, "rel_err": abs(fdv - adj) / max(abs(fdv), 1e-300)})
    s.set_coefficients(list(C))
    s.close()
    work = float(N) * nsteps
    t_grad = t_fwd + t_bwd
    return {
        "metric": "grid-pt·steps/s (gradient: forward with checkpoints + adjoint)", "value": work / t_grad,
        "unit": "grid-pt·steps/s", "n_gpus": 1, "steps": nsteps, "warmup": 1, "ms_per_step": t_grad * 1e3 / nsteps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(Ns), "L": list(Ls), "h": wl["h"], "T": wl["T"],
                   "checkpoint_every": wl["K"], "terms": len(terms), "loss": "mean squared mismatch vs target "
                   "from coefficients x (1 + 0.05 N(0,1)), seed 7", "ic": "glibc rand seed %d" % wl["seed"],
                   "l2": "state 1 MB: L2-resident (latency-bound regime)"},
        "cost_ratio": t_grad / t_plain, "seconds": {"plain_forward": t_plain, "forward_checkpointed": t_fwd,
                                                    "backward": t_bwd},
        "loss": L0, "fd_check": {"eps": 1e-6, "directions": 8, "max_rel_err": max(f["rel_err"] for f in fd),
                                 "cases": fd},
        "clocks": clk.summary(),
        "e2e": {"value": work / e2e_s, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": 2 * nN * 8 / nsteps,
                "d2h_bytes_per_step": 2 * nN * 8 / nsteps, "seconds": e2e_s},
    }


def run_bdf(args):
    """Stiff workload: 2D Brusselator u_t = 1 - 4u + u^2 v + lap u, v_t = 3u - u^2 v + 8 lap v
    on 256^2, L = 64, periodic 5-point finite differences, variable-order BDF at rtol = atol
    = 1e-6; initial state (1, 3) + U[-0.1, 0.1] from glibc rand() seed 3.  Warm-up
    [0, W tau], timed [W tau, (W+K) tau] (tau = 1); value = grid points x accepted steps /
    device seconds.  The linear solves are FFT-preconditioned GMRES (the reference's
    cuDSS is not available)."""
    import torch

    import rdcu_b200 as R
    from rdcu_b200.problems import brusselator_coupling_lines

    wl = WORKLOADS[args.workload]
    Ns, Ls = wl["Ns"], wl["Ls"]
    N = int(np.prod(Ns))
    nN = 2 * N
    terms = parse_terms(brusselator_coupling_lines())
    s = R.Solver(2, Ns, Ls, terms, method=R.METHOD_BDF, rtol=1e-6, atol=1e-6)
    y0 = R.random_ic(2, N, 0.2, 0.0, wl["seed"])
    y0[:N] += 1.0
    y0[N:] += 3.0
    T_A, T_B = args.warmup * wl["tau"], (args.warmup + args.steps) * wl["tau"]
    s.set_state(0.0, wl["h0"], y0.ctypes.data)
    s.solve(T_A, [])
    yA = np.empty(nN)
    D = np.empty(nN * 8)
    tA, hA, oA = s.get_state(yA.ctypes.data, D.ctypes.data)
    stream = torch.cuda.ExternalStream(s.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    lin0 = s.linear_stats()
    with ClockSampler(0) as clk:
        e0.record(stream)
        s.solve(T_B, [])
        e1.record(stream)
        e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    acc, att = s.counters()
    lin = [b - a for a, b in zip(lin0, s.linear_stats())]
    # e2e: the same window from host arrays through the C ABI, final state to the host
    w0 = time.perf_counter()
    s.set_state(tA, hA, yA.ctypes.data, oA, D.ctypes.data)
    s.solve(T_B, [])
    out = np.empty(nN)
    s.get_state(out.ctypes.data)
    e2e_s = time.perf_counter() - w0
    acc2, _ = s.counters()
    s.close()
    return {
        "metric": METRIC, "value": N * acc / sec, "unit": "grid-pt·steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(Ns), "L": list(Ls), "method": "BDF (NDF orders 1-5), FD",
                   "rtol": 1e-6, "atol": 1e-6, "window_sim_time": [T_A, T_B], "accepted_steps": acc,
                   "attempts": att, "linear_solver": "GMRES(40), FFT preconditioner",
                   "gmres": {"iterations": lin[0], "solves": lin[1], "restart_cycles": lin[2]},
                   "l2": "state 1 MB: L2-resident (latency-bound regime)"},
        "clocks": clk.summary(),
        "e2e": {"value": N * acc2 / e2e_s, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": 9 * nN * 8 / args.steps,
                "d2h_bytes_per_step": nN * 8 / args.steps, "seconds": e2e_s},
    }


def ensemble_members(wl):
    """Members of the ensemble workload: grid N x N with N drawn uniformly from the sizes,
    L = 0.78 N, CGLE b ~ U[0.5, 3], c ~ U[-2, 0] (numpy seed wl["seed"]); initial states
    uniform [-1, 1] from glibc rand() with seeds 0..members-1 (the reference's IC
    generator)."""
    rng = np.random.default_rng(wl["seed"])
    m = wl["members"]
    Ns = rng.choice(wl["sizes"], size=m)
    bs = rng.uniform(0.5, 3.0, size=m)
    cs = rng.uniform(-2.0, 0.0, size=m)
    mem = []
    for N, b, c in zip(Ns, bs, cs):
        N = int(N)
        lines = cgle_lines_bc(b, c)
        mem.append(dict(n=2, Ns=(N, N), Ls=(0.78 * N, 0.78 * N), terms=parse_terms(lines), rtol=1e-8, atol=1e-8))
    return mem


def cgle_lines_bc(b, c):
    from rdcu_b200.problems import cgle_coupling_lines

    return cgle_coupling_lines(2, b, c)


def run_ensemble(args, rank=0, world=1, local_rank=0):
    """Ensemble workload: 512 2D CGLE members of uneven size, adaptive DP45 at rtol = atol
    = 1e-8.  Warm-up [0, W tau] untimed, timed window [W tau, (W+K) tau] (tau = 0.1);
    value = sum over members of grid points x accepted steps / device seconds.  The
    instance-by-instance baseline runs a stratified sample of members (two per grid size)
    one after another through single handles over the same window and checks each
    member's accepted/attempt counts against the ensemble's; its rate is reported as
    baseline_sequential and the ratio as speedup_vs_sequential.  On N GPUs the members are
    dealt round-robin to the ranks (independent problems: no exchange); value = all
    members' work / the slowest rank's time (strong scaling of the fixed ensemble)."""
    import torch

    import rdcu_b200 as R

    wl = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    every = ensemble_members(wl)
    mine = [i for i in range(len(every)) if i % world == rank]
    mem = [every[i] for i in mine]
    m = len(mem)
    tau = wl["tau"]
    T_A, T_B = args.warmup * tau, (args.warmup + args.steps) * tau
    npts = np.array([x["Ns"][0] * x["Ns"][1] for x in mem], dtype=np.float64)
    ics = [R.random_ic(2, int(N), 2.0, 0.0, mine[i]) for i, N in enumerate(npts)]
    ens = R.Ensemble(mem, device=local_rank)
    for i in range(m):
        ens.set_state(i, 0.0, wl["h0"], ics[i].ctypes.data)
    tile = ens.tune()
    ens.solve(T_A)  # warm-up: the white-noise transient
    states = []
    for i in range(m):
        y = np.empty(2 * int(npts[i]))
        t, h = ens.get_state(i, y.ctypes.data)
        states.append((t, h, y))
        ens.set_state(i, t, h, y.ctypes.data)  # counters from the window start
    stream = torch.cuda.ExternalStream(ens.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        ens.solve(T_B)
        e1.record(stream)
        e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    cnt = np.array([ens.counters(i) for i in range(m)], dtype=np.float64)
    work = float(np.sum(cnt[:, 0] * npts))
    my_work = work
    if world > 1:
        sec, work = combine_ranks(sec, work, "cuda")
    # e2e: host states in, host states out, through the public API (same window)
    w0 = time.perf_counter()
    for i in range(m):
        ens.set_state(i, states[i][0], states[i][1], states[i][2].ctypes.data)
    ens.solve(T_B)
    outs = [np.empty(2 * int(N)) for N in npts]
    for i in range(m):
        ens.get_state(i, outs[i].ctypes.data)
    e2e_s = time.perf_counter() - w0
    e2e_work = my_work
    if world > 1:
        e2e_s, e2e_work = combine_ranks(e2e_s, my_work, "cuda")
    # instance-by-instance baseline on a stratified sample (of this rank's members)
    sample = []
    for N in wl["sizes"]:
        sample += [i for i in range(m) if mem[i]["Ns"][0] == N][:2]
    seq_s, seq_work = 0.0, 0.0
    for i in sample:
        s = R.Solver(2, mem[i]["Ns"], mem[i]["Ls"], mem[i]["terms"], rtol=1e-8, atol=1e-8)
        s.set_state(states[i][0], states[i][1], states[i][2].ctypes.data)
        torch.cuda.synchronize()
        st = torch.cuda.ExternalStream(s.stream)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        s.solve(T_B, [])
        a1.record(st)
        a1.synchronize()
        acc, att = s.counters()
        if (acc, att) != (int(cnt[i, 0]), int(cnt[i, 1])):
            raise RuntimeError("member %d: single handle took %d/%d steps, ensemble %d/%d" %
                               (i, acc, att, cnt[i, 0], cnt[i, 1]))
        seq_s += a0.elapsed_time(a1) / 1e3
        seq_work += acc * npts[i]
        s.close()
    seq_rate = seq_work / seq_s
    bytes_attempt = 41.0 * 8 * 2 * float(np.sum(npts))  # 41 state-sized arrays per DP45 attempt
    peak, peak_kind = load_peaks()
    attempts_batched = cnt[:, 1].max()
    achieved = bytes_attempt * attempts_batched / sec / 1e9
    ens.close()
    return {
        "metric": METRIC, "value": work / sec, "unit": "grid-pt·steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "members": len(every), "members_per_rank": m,
                   "parallelism": "members dealt to %d ranks" % world if world > 1 else "single",
                   "sizes": list(wl["sizes"]), "L": "0.78 N",
                   "coefficients": "b ~ U[0.5,3], c ~ U[-2,0] (numpy seed %d)" % wl["seed"],
                   "ic": "glibc rand seeds 0..%d, [-1,1]" % (m - 1), "rtol": 1e-8, "atol": 1e-8,
                   "window_sim_time": [T_A, T_B], "tau_per_step": tau, "tile_elems": tile,
                   "accepted_steps": int(cnt[:, 0].sum()), "attempts": int(cnt[:, 1].sum()),
                   "l2": "states 216 MB per array > L2 (no flush needed)"},
        "baseline_sequential": {"value": seq_rate, "unit": "grid-pt·steps/s", "sample_members": sample,
                                "seconds": seq_s, "note": "single handles one after another, same window"},
        "speedup_vs_sequential": (work / sec) / seq_rate,
        # per batched attempt: stages 2..7, each one kernel per line-length group of each
        # pass (fwd_x and inv_x by N[1], mid by N[0]), and the controller
        "gpu_launches": int(attempts_batched) * (6 * (2 * len({x["Ns"][1] for x in mem}) +
                                                      len({x["Ns"][0] for x in mem})) + 1),
        "clocks": clk.summary(),
        "e2e": {"value": e2e_work / e2e_s, "unit": "grid-pt·steps/s",
                "h2d_bytes_per_step": 16.0 * float(np.sum(npts)) / args.steps,
                "d2h_bytes_per_step": 32.0 * float(np.sum(npts)) / args.steps, "seconds": e2e_s},
        "roofline": {"bound": "hbm", "kernel": "batched DP45 attempt (all passes)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_attempt": bytes_attempt, "batched_attempts": int(attempts_batched)},
    }


def line_frames(wl, count, device):
    """Synthetic 3D CGLE-like frames with vortex lines (no dataset exists): the phase is a
    sum of wl["terms"] terms atan2(sin(2 pi (x_b - q)/N_b), sin(2 pi (x_a - p)/N_a)) --
    four periodic lines along the third axis each, wobbling along it and drifting
    wl["drift"] cells per frame -- plus Gaussian phase noise; amplitude 1 + U[0, 0.2].
    Returns a (count, 2*N) float64 tensor on `device` (u block, v block per frame)."""
    import torch

    Ns = wl["Ns"]
    rng = np.random.default_rng(wl["seed"])
    g = torch.meshgrid(*[torch.arange(n, dtype=torch.float64, device=device) for n in Ns], indexing="ij")
    terms = []
    for _ in range(wl["terms"]):
        ax = int(rng.integers(3))
        a, b = [x for x in range(3) if x != ax]
        terms.append((ax, a, b, rng.uniform(0, Ns[a]), rng.uniform(0, Ns[b]), *(rng.normal(size=2) * wl["drift"]),
                      rng.uniform(0, 2.5), rng.uniform(0, 2 * np.pi)))
    gen = torch.Generator(device=device)
    gen.manual_seed(wl["seed"])
    n = int(np.prod(Ns))
    out = torch.empty((count, 2 * n), dtype=torch.float64, device=device)
    for k in range(count):
        th = torch.zeros(Ns, dtype=torch.float64, device=device)
        for ax, a, b, p0, q0, vp, vq, amp, ph in terms:
            s_ = 2 * np.pi * g[ax] / Ns[ax] + ph
            p = p0 + vp * k + amp * torch.sin(s_)
            q = q0 + vq * k + amp * torch.cos(s_)
            th += torch.atan2(torch.sin(2 * np.pi * (g[b] - q) / Ns[b]), torch.sin(2 * np.pi * (g[a] - p) / Ns[a]))
        th += wl["noise"] * torch.randn(Ns, dtype=torch.float64, device=device, generator=gen)
        r = 1.0 + 0.2 * torch.rand(Ns, dtype=torch.float64, device=device, generator=gen)
        out[k, :n] = (r * torch.cos(th)).reshape(-1)
        out[k, n:] = (r * torch.sin(th)).reshape(-1)
    return out


def lines_cpu_sample(wl, frames_host, count):
    """The oracle (numpy/scipy, one thread) on `count` frames: phase, lines, correlate
    with the previous frame.  Returns seconds per frame."""
    from oracle import lines as ol

    Ns, Ls = wl["Ns"], wl["Ls"]
    prev = ol.findlines(ol.phase(frames_host[0], Ns), Ns, Ls)
    t0 = time.perf_counter()
    for k in range(1, count + 1):
        cur = ol.findlines(ol.phase(frames_host[k], Ns), Ns, Ls)
        ol.correlate(prev, cur, Ns, Ls)
        prev = cur
    return (time.perf_counter() - t0) / count


def run_lines(args, rank=0, world=1, local_rank=0):
    """Defect-line workload (the reference's makelines.py per-frame work): for each frame
    of a sequence of 128^3 2-field states, the phase, plaquette windings, line cubes,
    their components and edge lists (findlines), and the distance matrix to the previous
    frame's components (correlate).  A bench step is wl["frames_per_step"] frames, taken
    in turn from a ring of wl["ring"] distinct frames (1.6 GB, beyond L2); value =
    frames/s.  ``value`` runs on frames resident in HBM (edge lists stay on the device,
    the small distance matrix comes back); ``e2e`` starts from pinned host frames and
    brings every frame's edge list and distance matrix to the host through the public
    API, each frame's copy staged (rdcu_lines_prefetch) while the previous one is found.  On N GPUs each rank processes its own frame sequence (independent frames: no
    exchange)."""
    import torch

    from rdcu_b200.lines import STATE, Lines

    wl = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    Ns, Ls = wl["Ns"], wl["Ls"]
    N = int(np.prod(Ns))
    W, K, F, R = args.warmup, args.steps, wl["frames_per_step"], wl["ring"]
    frames = line_frames(dict(wl, seed=wl["seed"] + rank), R, "cuda")
    hs = [Lines(Ns, Ls, local_rank), Lines(Ns, Ls, local_rank)]

    def step(k, src):
        cur, prev = hs[k % 2], hs[(k - 1) % 2]
        cur.find(src[k % R], STATE)
        return cur.correlate(prev)

    hs[0].find(frames[0], STATE)
    for k in range(1, W * F + 1):
        step(k, frames)
    k0, k1 = W * F + 1, (W + K) * F + 1
    launches0 = sum(h.info()[2] for h in hs)
    streams = [torch.cuda.ExternalStream(h.stream) for h in hs]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    comps, cubes = [], []
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        e0.record(streams[k0 % 2])
        for k in range(k0, k1):
            d = step(k, frames)
            comps.append(d.shape[0])
            cubes.append(hs[k % 2].counts[0])
        e1.record(streams[(k1 - 1) % 2])
        e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    launches = sum(h.info()[2] for h in hs) - launches0
    # one find alone, CUDA events on its stream, and its passes (rdcu_lines_profile)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    f0.record(streams[0])
    for r in range(8):
        hs[0].find(frames[r], STATE)
    f1.record(streams[0])
    f1.synchronize()
    find_s = f0.elapsed_time(f1) / 1e3 / 8
    passes = hs[0].profile(frames[W + 1], STATE, reps=10)
    top = max(passes, key=lambda p: p[1])
    work = float(K * F)
    if world > 1:
        sec, work = combine_ranks(sec, work, "cuda")
    # e2e: pinned host frames in, edge lists and distance matrices out
    host = frames.cpu().pin_memory()
    torch.cuda.synchronize()
    hs[(k0 - 1) % 2].find(host[(k0 - 1) % R], STATE)
    hs[k0 % 2].prefetch(host[k0 % R], STATE)
    w0 = time.perf_counter()
    out_bytes = 0
    for k in range(k0, k1):
        cur, prev = hs[k % 2], hs[(k - 1) % 2]
        if k + 1 < k1:  # frame k+1 copies into the previous frame's handle while k is found
            prev.prefetch(host[(k + 1) % R], STATE)
        cur.find(None, STATE)
        d = cur.correlate(prev)
        xyz, off = cur.edges()
        out_bytes += xyz.nbytes + off.nbytes + d.nbytes
    e2e_s = time.perf_counter() - w0
    e2e_work = float(K * F)
    if world > 1:
        e2e_s, e2e_work = combine_ranks(e2e_s, e2e_work, "cuda")
    peak, peak_kind = load_peaks()
    find_bytes = 40.0 * N  # state 16 B read; phase 8 B written, 8 B read; face, mark, node map 8 B
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        per = lines_cpu_sample(wl, host.numpy(), 2)
        cpu = {"value": 1.0 / per, "unit": "frames/s", "cores": 1, "kind": "port",
               "sample": "oracle/lines.py (numpy/scipy, one thread) on 2 frames: phase, lines, correlate"}
    for h in hs:
        h.close()
    return {
        "metric": "frames/s", "value": work / sec, "unit": "frames/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": sec * 1e3 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(Ns), "L": list(Ls), "frames_per_step": F,
                   "frames": "synthetic vortex-line states, %d terms (4 lines each), phase noise %g, drift %g "
                             "cells/frame, seed %d, ring of %d" % (wl["terms"], wl["noise"], wl["drift"],
                                                                  wl["seed"], R),
                   "mean_line_cubes": float(np.mean(cubes)), "mean_components": float(np.mean(comps)),
                   "parallelism": "independent frame sequences per rank" if world > 1 else "single",
                   "l2": "ring of %d distinct 33.5 MB frames (1.6 GB > L2), no flush needed" % R},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "e2e": {"value": e2e_work / e2e_s, "unit": "frames/s", "h2d_bytes_per_step": 16.0 * N * F,
                "d2h_bytes_per_step": out_bytes / K, "seconds": e2e_s},
        "roofline": {"bound": "hbm", "kernel": "rdcu_lines_find pass '%s'" % top[0],
                     "achieved": top[2] / (top[1] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": top[2] / (top[1] / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                     "traffic": NCU_TRAFFIC_LINES.get(top[0]), "algorithmic_bytes_per_launch": top[2],
                     "launch_ms": top[1], "find_ms": find_s * 1e3,
                     "find_achieved_GBps": find_bytes / find_s / 1e9,
                     "passes": [{"name": a, "ms": b, "bytes": c, "GBps": c / (b / 1e3) / 1e9 if b > 0 else None,
                                 "share": b / sum(p[1] for p in passes)} for a, b, c in passes]},
        "cpu_baseline": cpu,
    }


def cli_run(exe, wl):
    """One CLI run of the workload's command line in a scratch directory (coupling file:
    the reference notebook's CGLE).  Returns the integration-only rate from the .out
    progress lines (N x difference of the cumulative steps / difference of the elapsed
    seconds between the first and last output), the run's own totals and wall time."""
    Ns = wl["Ns"]
    N = int(np.prod(Ns))
    with tempfile.TemporaryDirectory() as wd:
        fb = os.path.join(wd, "cli")
        open(fb + "coupling.dat", "w").write("\n".join(cgle_lines(len(Ns))) + "\n")
        cmd = [exe] + shlex.split(wl["cli"]) + [fb]
        w0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
        wall = time.perf_counter() - w0
        out = open(fb + ".out").read() if os.path.exists(fb + ".out") else ""
        states = os.path.getsize(fb + "states.dat") if os.path.exists(fb + "states.dat") else 0
    prog = []
    for line in out.splitlines():
        f = line.split("\t")
        if len(f) >= 5 and re.fullmatch(r"[0-9.]+", f[0]):
            prog.append((float(f[1]), int(f[4])))
    m = re.search(r"steps: (\d+)", out)
    rt = re.search(r"runtime: ([0-9.]+)", out)
    if r.returncode != 0 or len(prog) < 2 or not m:
        return None, "rc %d, %d progress lines: %s" % (r.returncode, len(prog), (r.stderr or r.stdout)[-200:])
    (e0, s0), (e1, s1) = prog[0], prog[-1]
    return {"value": N * (s1 - s0) / (e1 - e0), "steps": int(m.group(1)), "window_steps": s1 - s0,
            "window_s": e1 - e0, "runtime_s": float(rt.group(1)) if rt else None, "wall_s": wall,
            "outputs": len(prog), "states_bytes": states, "command": " ".join(shlex.quote(c) for c in cmd)}, None


def run_cli(args, impl):
    """CLI workloads: the same command line through this package's rdcu CLI (ours) or the
    reference's own build (reference arm), outputs included; value from the .out
    progress lines, as for the reference (the integration between the first and the
    last output, set-up excluded, output writes included)."""
    wl = WORKLOADS[args.workload]
    if impl == "reference":
        exe, why = reference_binary()
        if exe is None:
            return {"impl": "reference", "unavailable": why}
    else:
        from rdcu_b200 import CLI_PATH

        exe = CLI_PATH
    with ClockSampler(0) as clk:
        res, err = cli_run(exe, wl)
    if res is None:
        line = {"metric": METRIC, "unavailable": "CLI run failed: " + err}
        if impl == "reference":
            line["impl"] = "reference"
        return line
    line = {
        "metric": METRIC, "value": res["value"], "unit": "grid-pt·steps/s", "n_gpus": 1,
        "steps": res["outputs"] - 1, "warmup": 0, "ms_per_step": res["window_s"] * 1e3 / max(1, res["outputs"] - 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "command": res["command"], "accepted_steps": res["steps"],
                   "window_steps": res["window_steps"], "outputs": res["outputs"],
                   "states_bytes": res["states_bytes"], "runtime_s": res["runtime_s"], "wall_s": res["wall_s"],
                   "step": "one output interval of the run (dt = 1)"},
        "e2e": {"value": res["value"], "unit": "grid-pt·steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": res["states_bytes"] / max(1, res["outputs"]),
                "note": "CLI process: outputs written to states.dat inside the window"},
        "gpu_launches": None,
        "clocks": clk.summary(),
    }
    if impl == "reference":
        line["impl"] = "reference"
        line["cpu_baseline"] = {"value": res["value"], "unit": "grid-pt·steps/s", "cores": 1, "kind": "reference",
                                "sample": "the reference's own CLI build on the same command line"}
    return line


def run_lines_reference(args):
    """Reference arm of the defect-line workload: the reference's line tracker is Python
    (makelines.py, numpy + torch + networkx) that is not on the GPU box, so its CPU
    restatement oracle/lines.py times a bounded sample of the same frames (phase, lines,
    correlate per frame, one thread)."""
    import torch

    wl = WORKLOADS[args.workload]
    n = 4
    frames = line_frames(wl, n + 1, "cuda" if torch.cuda.is_available() else "cpu").cpu().numpy()
    per = lines_cpu_sample(wl, frames, n)
    value = 1.0 / per
    return {
        "impl": "reference", "metric": "frames/s", "value": value, "unit": "frames/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3 * wl["frames_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(wl["Ns"]), "L": list(wl["Ls"])},
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": 1, "kind": "port",
                         "sample": "oracle/lines.py on %d frames of the workload (phase, findlines, correlate each)"
                                   % n},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's makelines.py cannot run on the box; the oracle builds the neighbour graph from "
                "the grid, faster than the reference's all-pairs test, so this arm overstates the reference",
    }


def launches_per_attempt_of(name, names=()):
    """Launches of a pass in one DP45 attempt (stages 2-7): the forward and inverse
    x passes of stages 2-6 five times and their stage-7 forms once; the passes between
    them (axis 0, and axis 1 unless the x passes do it) six times.  With fused x passes
    (`inv_fwd_row` among `names`: the inverse pass of stages 2-5 also does the next
    stage's forward pass) the attempt runs stage 2's forward pass, the fused pass four
    times, stage 6's inverse pass and stage 7's two x passes; the forward pass of stage 4
    (`fwd_x`) is listed but does not run."""
    if "inv_fwd_row" in names:
        fused = {"fwd_x_stage2": 1, "inv_fwd_row": 4, "inv_x_dictionary": 1, "fwd_x_stage7": 1,
                 "inv_x_stage7": 1, "fwd_x": 0}
        if name in fused:
            return fused[name]
        return 6
    if name.endswith("_stage7"):
        return 1
    if name.startswith("fwd_") or name.startswith("inv_"):
        return 5
    return 6


def cpu_baseline(Ns, Ls, y, t, h):
    """One DP45 attempt of the same workload on the host cores (oracle port)."""
    from oracle import cpu_port

    ncores = os.cpu_count() or 1
    t0 = time.perf_counter()
    acc = cpu_port.dp45_attempts(Ns, Ls, y, h, attempts=1, workers=ncores)
    sec = time.perf_counter() - t0
    N = int(np.prod(Ns))
    return {"value": N * max(acc, 1) / sec, "unit": "grid-pt·steps/s", "cores": ncores, "kind": "port",
            "sample": "1 DP45 attempt (6 RHS) of the %s CGLE from the state at the window start, "
                      "numpy + scipy.fft with %d workers; %.1f s" % ("x".join(map(str, Ns)), ncores, sec)}


# ----------------------------------------------------------------------------- reference arm
def reference_binary():
    """The reference's own build, compiled beforehand from its sources by
    oracle/build_ref.sh (the build step does it where the sources are present)."""
    p = os.path.join(ROOT, "oracle", "_ref", "rdcu_ref")
    if os.path.exists(p):
        return p, None
    return None, "reference binary oracle/_ref/rdcu_ref not built (oracle/build_ref.sh builds it from the sources)"


def run_reference(args):
    if args.workload.startswith("adjoint"):
        return {"impl": "reference", "unavailable": "the reference computes no gradients (no adjoint to time)"}
    if args.workload.startswith("bdf"):
        return {"impl": "reference", "unavailable": "the reference's BDF path needs cuDSS, which is not installed "
                "in this image (no cudss.h or libcudss)"}
    if args.workload.startswith("ensemble"):
        return {"impl": "reference", "unavailable": "the reference has no ensemble; its one-problem-per-process "
                "rate is the cgle2d workloads' reference arm, and the instance-by-instance baseline of this "
                "workload is reported by our arm"}
    if args.workload.startswith("lines"):
        return run_lines_reference(args)
    if args.workload.startswith("cli"):
        return run_cli(args, "reference")
    exe, why = reference_binary()
    if exe is None:
        return {"impl": "reference", "unavailable": why}
    wl = WORKLOADS[args.workload]
    Ns, Ls = wl["Ns"], wl["Ls"]
    N = int(np.prod(Ns))
    T_A = args.warmup * TAU
    # The reference times from program start (CUDA and cuFFT set-up included), so the
    # rate comes from the progress lines of one run, set-up outside the window:
    # 2D: outputs every T_A, rate between the progress lines at T_A and at the end (the
    #     outputs of these small grids cost nothing noticeable);
    # 3D: outputs only at the window's two ends (below); grids up to 2M points use a
    #     window ten times the bench's (the reference then integrates ~15 s in it).
    mult = 10 if (len(Ns) == 3 and N <= (1 << 21)) else 1
    T_B = (args.warmup + mult * args.steps) * TAU

    def one(T, dt):
        with tempfile.TemporaryDirectory() as wd:
            fb = os.path.join(wd, "bench")
            open(fb + "coupling.dat", "w").write("\n".join(cgle_lines(len(Ns))) + "\n")
            # -D1 (the reference writes times.dat unconditionally at outputs, so -D0
            # crashes it); first step h0 as in our arm
            cmd = [exe, "-n", "2", "-N", ",".join(map(str, Ns)), "-L", ",".join("%g" % l for l in Ls),
                   "-A", "2", "-s", str(wl["seed"]), "-t", repr(T), "-d", "%r,%r" % (dt, wl["h0"]), "-D1", fb]
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
            out = open(fb + ".out").read() if os.path.exists(fb + ".out") else ""
            m = re.search(r"steps: (\d+)", out)
            rt = re.search(r"runtime: ([0-9.]+)", out)
            prog = []
            for line in out.splitlines():
                f = line.split("\t")
                if len(f) >= 5 and re.fullmatch(r"[0-9.]+", f[0]):
                    prog.append((float(f[1]), int(f[4])))
            return (int(m.group(1)) if m else -1, float(rt.group(1)) if rt else -1.0, prog, r.returncode,
                    " ".join(shlex.quote(c) for c in cmd))

    if len(Ns) == 2:
        sB, rB, prog, cB, cmdB = one(T_B, T_A)
        if cB != 0 or len(prog) < 2:
            return {"impl": "reference", "unavailable": "reference run failed (rc %d, %d outputs)" % (cB, len(prog))}
        (e0, s0), (e1, s1) = prog[0], prog[-1]
        value = N * (s1 - s0) / (e1 - e0)
        window_steps, window_s = s1 - s0, e1 - e0
        sample = ("reference nvcc sm_100a build (cuFFT/cuBLAS), one run to t=%g with outputs every %g; rate "
                  "between the progress lines at t=%g and t=%g (%d steps, %.3f s), set-up excluded"
                  % (T_B, T_A, T_A, T_B, window_steps, window_s))
    else:
        # one run whose only outputs are the window's two ends: outputs every W = T_B - T_A
        # from t = W to t = 2 W, the rate between those two progress lines (the per-step
        # cost does not depend on where the window sits; set-up and the first output's
        # file write are outside it, the second output's write inside it)
        W = T_B - T_A
        T_A, T_B = W, 2 * W
        sB, rB, prog, cB, cmdB = one(T_B, W)
        if cB != 0 or len(prog) < 2:
            return {"impl": "reference", "unavailable": "reference run failed (rc %d, %d outputs)" % (cB, len(prog))}
        (e0, s0), (e1, s1) = prog[0], prog[-1]
        value = N * (s1 - s0) / (e1 - e0)
        window_steps, window_s = s1 - s0, e1 - e0
        sample = ("reference nvcc sm_100a build (cuFFT/cuBLAS), one run to t=%g with outputs every %g; rate "
                  "between the progress lines at t=%g and t=%g (%d steps, %.3f s), set-up excluded"
                  % (T_B, W, T_A, T_B, window_steps, window_s))
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "grid-pt·steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": window_s * 1e3 / (mult * args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(Ns), "L": list(Ls), "window_sim_time": [T_A, T_B],
                   "accepted_steps": window_steps, "window_s": window_s, "command": cmdB},
        "cpu_baseline": {"value": value, "unit": "grid-pt·steps/s", "cores": 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU implementation of the path; its own GPU build is the reference arm",
    }


# The other targets, measured by their own workloads in separate processes (each holds its
# own device memory) and summarised on the default line: the ensemble against its
# instance-by-instance baseline, the adjoint's cost ratio and finite-difference check, the
# BDF rate.  Each record keeps its run's clocks.
SECONDARY = [
    ("ensemble_cgle2d_512", ["--steps", "20", "--warmup", "3"],
     lambda r: {"value": r["value"], "unit": r["unit"], "baseline_sequential": r["baseline_sequential"]["value"],
                "speedup_vs_sequential": r["speedup_vs_sequential"], "members": r["config"]["members"],
                "window_sim_time": r["config"]["window_sim_time"], "e2e": r["e2e"]["value"],
                "roofline_frac": r["roofline"]["frac"]}),
    ("adjoint_cgle2d_256", ["--steps", "1", "--warmup", "3"],
     lambda r: {"value": r["value"], "unit": r["unit"], "cost_ratio": r["cost_ratio"],
                "fd_max_rel_err": r["fd_check"]["max_rel_err"], "fd_directions": r["fd_check"]["directions"],
                "seconds": r["seconds"], "steps": r["steps"]}),
    ("bdf_brusselator_256", ["--steps", "40", "--warmup", "4"],
     lambda r: {"value": r["value"], "unit": r["unit"], "accepted_steps": r["config"]["accepted_steps"],
                "window_sim_time": r["config"]["window_sim_time"], "gmres": r["config"]["gmres"],
                "e2e": r["e2e"]["value"]}),
]


def secondary_records():
    out = {}
    for wl, extra, pick in SECONDARY:
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", wl, "--no-cpu-baseline"] + extra
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            line = json.loads(r.stdout.strip().splitlines()[-1])
            rec = pick(line)
            rec["clocks"] = line.get("clocks")
            rec["command"] = "python bench.py --workload %s --no-cpu-baseline %s" % (wl, " ".join(extra))
            out[wl] = rec
        except Exception as e:  # a failed record is reported, not fatal to the headline
            out[wl] = {"error": "%s: %s" % (type(e).__name__, str(e)[:300])}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cgle3d_256", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the ensemble, adjoint and BDF records of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.workload.startswith("adjoint"):
        line = run_adjoint(args) if rank == 0 else None
    elif args.workload.startswith("ensemble"):
        line = run_ensemble(args, rank, world, local_rank)
    elif args.workload.startswith("bdf"):
        line = run_bdf(args) if rank == 0 else None
    elif args.workload.startswith("lines"):
        line = run_lines(args, rank, world, local_rank)
    elif args.workload.startswith("cli"):
        line = run_cli(args, "ours") if rank == 0 else None
    else:
        line = run_ours(args, rank, world, local_rank)
        if rank == 0 and world == 1 and args.workload == "cgle3d_256" and not args.no_secondary:
            line["secondary"] = secondary_records()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
