"""Oracle: emulation of the reference driver (``main`` and ``step_eval``).

Test infrastructure only (see ``oracle/__init__``).  Restates rdcu.cu:863-1198 (initial
conditions, output files, initial outputs, integration) and ``step_eval``
(rdcu.cu:252-341), writing the same binary files so the CLI of the library can be
compared with it file by file.  Progress lines carry wall-clock timings and are not
reproduced; ``.out`` only receives the final ``steps:`` line.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

from . import bdf as obdf
from . import dp45 as odp
from . import fd as ofd
from . import spectral as osp
from .problem import Problem, Term, glibc_uniform_ic, read_fs, t_eval_grid


@dataclass
class RunConfig:
    """The option values of the reference CLI (defaults from rdcu.cu:603-607)."""

    n: int = 1
    Ns: Tuple[int, ...] = (128,)
    Ls: Tuple[float, ...] = (1.0,)
    terms: List[Term] = field(default_factory=list)
    A: float = 1e-3
    A0: float = 0.0
    t1: float = 1e2
    dt: float = 1e0
    h: float = 0.0
    hmin: float = 0.0
    hmax: float = math.inf
    seed: int = 1
    dense: int = 1
    stiff: bool = False
    fixed: bool = False
    reload: bool = False
    rtol: float = 1e-8
    atol: float = 1e-8
    max_attempts: int | None = None
    linear: str = "lu"  # BDF linear solver: "lu" (direct, as cuDSS) or "gmres" (oracle.gmres)


def run(filebase: str, cfg: RunConfig) -> dict:
    """Runs the emulated reference; returns a summary dict (steps, attempts, t, h)."""
    prob = Problem(cfg.n, tuple(cfg.Ns), tuple(cfg.Ls), list(cfg.terms))
    n, N, nN = prob.n, prob.N, prob.n * prob.N
    st = ofd.stencils(prob) if cfg.stiff else None

    def dydt_full(t, y):
        if cfg.stiff:
            Yr = ofd.fd_Y(y, prob, st)
            return osp.dictionary_rhs(Yr, prob), Yr.astype(np.complex128)
        return osp.rhs(y, prob, return_Y=True)

    def dydt(t, y):
        return dydt_full(t, y)[0]

    def jac(t, y):
        return ofd.jacobian(y, prob, st)

    h = cfg.h
    if h <= 0.0:
        h = cfg.dt if cfg.fixed else cfg.dt / 100
    t = 0.0
    order = 0
    loaded = reloaded = False
    y = None
    D_re = []
    out = open(filebase + ".out", "w")
    ic = filebase + "ic.dat"
    if os.path.exists(ic):
        loaded = True
        raw = np.fromfile(ic, np.float64)
        if raw.size >= nN:
            y = raw[:nN].copy()
        else:
            loaded = False
    fs = filebase + "fs.dat"
    if cfg.reload and os.path.exists(fs):
        reloaded = loaded = True
        yv, tv, hv, ordv, Dv = read_fs(fs, nN, cfg.stiff)
        y, t, h, order, D_re = yv, tv, hv, ordv, Dv
    if not reloaded and not loaded:
        y = glibc_uniform_ic(n, N, cfg.A, cfg.A0, cfg.seed)
        with open(fs, "wb") as fh:
            fh.write(y.tobytes()); fh.write(np.float64(t).tobytes()); fh.write(np.float64(h).tobytes())

    wt = "ab" if loaded else "wb"
    files = {}
    if cfg.dense >= 1:
        for k in ("steps", "times", "states"):
            files[k] = open(filebase + k + ".dat", wt)
    if cfg.dense >= 2:
        files["f"] = open(filebase + "f.dat", wt)
    if cfg.dense >= 3:
        files["Y"] = open(filebase + "Y.dat", wt)
    if cfg.dense >= 4:
        for k in ("rows", "cols", "vals"):
            files[k] = open(filebase + k + ".dat", wt)

    t0 = t
    t_eval = t_eval_grid(t, cfg.t1, cfg.dt)

    def write_jac(yv, tt):
        if cfg.stiff:
            r, c, v = jac(tt, yv)
        else:
            # without -S the reference's stencil tables are empty: rows are all zero
            r, c, v = np.zeros(nN + 1, np.int32), np.zeros(0, np.int32), np.zeros(0)
        files["rows"].write(np.asarray(r, np.int32).tobytes())
        files["cols"].write(np.asarray(c, np.int32).tobytes())
        files["vals"].write(np.asarray(v, np.float64).tobytes())

    if cfg.dense >= 1 and not cfg.reload:
        files["states"].write(y.tobytes())
        files["times"].write(np.float64(t).tobytes())
    if cfg.dense >= 2 and not cfg.reload:
        f0, Y0 = dydt_full(t, y)
        files["f"].write(f0.tobytes())
        if cfg.dense >= 3:
            files["Y"].write(np.asarray(Y0, np.complex128).tobytes())
        if cfg.dense >= 4 and cfg.stiff:
            write_jac(y, t)

    state = {"steps": 0, "eval_i": 0, "attempts": 0}
    if cfg.stiff:
        D0 = [y] + list(D_re)
        stepper = obdf.BDF(D0, order, cfg.atol, cfg.rtol, cfg.fixed, dydt, jac, linear=cfg.linear)
    else:
        stepper = odp.DP45(y, cfg.atol, cfg.rtol, cfg.fixed, dydt)

    def step_eval(tt, hh, yy, success):
        state["attempts"] += 1
        if cfg.dense >= 1:
            files["steps"].write(np.float64(hh).tobytes())
        if not success:
            return
        state["steps"] += 1
        ev = False
        while state["eval_i"] < len(t_eval) and tt >= t_eval[state["eval_i"]]:
            te = t_eval[state["eval_i"]]
            ye = stepper.eval(tt, hh, te) if cfg.stiff else stepper.eval(tt, te)
            if cfg.dense >= 1:
                files["states"].write(ye.tobytes())
            if cfg.dense >= 2:
                fe, Ye = dydt_full(te, ye)
                files["f"].write(fe.tobytes())
                if cfg.dense >= 3:
                    files["Y"].write(np.asarray(Ye, np.complex128).tobytes())
            if cfg.dense >= 4:
                write_jac(ye, te)
            if cfg.dense >= 1:
                files["times"].write(np.float64(te).tobytes())
            state["eval_i"] += 1
            ev = True
        if ev:
            out.write("%.3f\t%1.3e\t%1.3e\t%f\t%i\t\n" % ((tt - t0) / (cfg.t1 - t0), 0.0, 0.0,
                                                         hh, state["steps"]))
            with open(fs, "wb") as fh:
                fh.write(yy.tobytes()); fh.write(np.float64(tt).tobytes())
                fh.write(np.float64(hh).tobytes())
                if cfg.stiff:
                    fh.write(np.int32(stepper.order).tobytes())
                    for i in range(1, stepper.order + 1):
                        fh.write(stepper.D[i].tobytes())

    t, h = stepper.run(t, h, cfg.hmin, cfg.hmax, cfg.t1, step_eval, cfg.max_attempts)
    out.write("\nsteps: %i\n" % state["steps"])
    out.close()
    for fh in files.values():
        fh.close()
    return {"steps": state["steps"], "attempts": state["attempts"], "t": t, "h": h,
            "order": getattr(stepper, "order", None), "linear": getattr(stepper, "lin_stats", None)}


def config_from_argv(argv: List[str]):
    """Option parsing of rdcu.cu:603-731 (getopt "hvFRSn:N:L:c:A:t:d:s:D:g:r:a:", GNU
    argument permutation, the last positional argument is FILEBASE).  Returns
    (RunConfig, filebase, help, verbose); coupling terms from ``-c`` only (the caller
    appends FILEBASEcoupling.dat terms, rdcu.cu:822-837)."""
    import getopt

    from .problem import c_atof, c_atoi, parse_term, _strtok

    opts, rest = getopt.gnu_getopt(argv, "hvFRSn:N:L:c:A:t:d:s:D:g:r:a:")
    cfg = RunConfig()
    Ns = [128, 128, 128]
    Ls = [1.0, 1.0, 1.0]
    ndim = 1
    nL = 0
    helpf = True
    verbose = False
    for o, a in opts:
        if o == "-h":
            helpf = True
        elif o == "-v":
            verbose = True
        elif o == "-F":
            cfg.fixed = True
        elif o == "-R":
            cfg.reload = True
        elif o == "-S":
            cfg.stiff = True
        elif o == "-n":
            cfg.n = c_atoi(a)
        elif o == "-N":
            vals = [c_atoi(t) for _, t in _strtok(a, ",")][:3]
            ndim = len(vals)
            Ns[:len(vals)] = vals
        elif o == "-L":
            vals = [c_atof(t) for _, t in _strtok(a, ",")]
            vals = vals[: max(0, 3 - nL)]
            Ls[nL:nL + len(vals)] = vals
            nL += len(vals)
        elif o == "-c":
            t = parse_term(a)
            if t is not None:
                cfg.terms.append(t)
        elif o == "-A":
            vals = [c_atof(t) for _, t in _strtok(a, ",")][:4]
            cfg.A = vals[0] if vals else 0.0
            if len(vals) > 1:
                cfg.A0 = vals[1]
        elif o == "-t":
            cfg.t1 = c_atof(a)
        elif o == "-d":
            vals = [c_atof(t) for _, t in _strtok(a, ",")][:4]
            cfg.dt = vals[0]
            if len(vals) > 1:
                cfg.h = vals[1]
            if len(vals) > 2:
                cfg.hmin = vals[2]
            if len(vals) > 3:
                cfg.hmax = vals[3]
        elif o == "-s":
            cfg.seed = c_atoi(a)
        elif o == "-D":
            cfg.dense = c_atoi(a)
        elif o == "-r":
            cfg.rtol = c_atof(a)
        elif o == "-a":
            cfg.atol = c_atof(a)
    filebase = None
    for r in rest:
        filebase = r
        helpf = False
    cfg.Ns = tuple(Ns[:ndim])
    cfg.Ls = tuple(Ls[:ndim])
    return cfg, filebase, helpf, verbose
