"""rdcu_b200 -- B200-native FP64 dictionary reaction-diffusion solver.

Python binding of the C ABI in ``include/rdcu.h`` (``librdcu.so``, built in-tree by
``rdcu_b200.build``).  The reference drives its solver through the ``rdcu`` command
line (its Python post-processing runs ``./rdcu`` with ``os.system``,
reference makelines.py:260-268); the same CLI is built here as ``rdcu_b200/bin/rdcu``.
This module exposes the library itself to Python: problem handles, RHS and Jacobian
evaluation, stepping, dense output and whole integrations with an output callback.

Buffers are passed as integer addresses (host or device, for example
``torch.Tensor.data_ptr()`` of a float64 CUDA tensor) or as the array or tensor itself,
which keeps it alive for the call (see ``_addr``).  There is no CPU fallback: loading
fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import numbers
import os
from typing import Callable, List, Optional, Sequence, Union

# a buffer argument: an integer address, a numpy array or a tensor (see _addr)
Buffer = Union[int, "numpy.ndarray", "torch.Tensor"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librdcu.so")
CLI_PATH = os.path.join(HERE, "bin", "rdcu")

RDCU_OK = 0
RDCU_ERR_INVALID = -1
RDCU_ERR_CUDA = -2
RDCU_ERR_UNSUPPORTED = -3
RDCU_ERR_TIMEOUT = -4
RDCU_ERR_NOMEM = -5
RDCU_ERR_NUMERIC = -6
RDCU_ERR_STATE = -7
RDCU_ERR_CALLBACK = -8

METHOD_DP45 = 0
METHOD_BDF = 1

EV_ATTEMPT = 0
EV_EVAL = 1
EV_CHECKPOINT = 2

# exported entry points of include/rdcu.h
EXPORTS = [
    "rdcu_create", "rdcu_destroy", "rdcu_set_state", "rdcu_get_state", "rdcu_get_info",
    "rdcu_rhs", "rdcu_jac", "rdcu_step", "rdcu_eval", "rdcu_solve", "rdcu_get_counters", "rdcu_get_linear_stats",
    "rdcu_memcpy", "rdcu_advance", "rdcu_random_ic", "rdcu_profile_passes", "rdcu_rhs_noalloc",
    "rdcu_set_coefficients", "rdcu_adjoint_forward", "rdcu_adjoint_backward",
    "rdcu_ensemble_create", "rdcu_ensemble_destroy", "rdcu_ensemble_set_state", "rdcu_ensemble_get_state",
    "rdcu_ensemble_solve", "rdcu_ensemble_counters", "rdcu_ensemble_tune", "rdcu_ensemble_info",
    "rdcu_ensemble_last_error", "rdcu_lines_create", "rdcu_lines_destroy", "rdcu_lines_find", "rdcu_lines_prefetch", "rdcu_lines_edges",
    "rdcu_lines_cubes", "rdcu_lines_correlate", "rdcu_lines_correlate_sets", "rdcu_lines_profile", "rdcu_lines_info",
    "rdcu_lines_last_error", "rdcu_error_string", "rdcu_last_error",
]
_STRING_RESULTS = ("rdcu_error_string", "rdcu_last_error", "rdcu_ensemble_last_error", "rdcu_lines_last_error")


class RdcuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("rdcu error %d: %s" % (code, msg))
        self.code = code


class rdcu_spec(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("ndim", ctypes.c_int), ("Ns", ctypes.c_int * 3),
        ("Ls", ctypes.c_double * 3), ("nterms", ctypes.c_int),
        ("C", ctypes.POINTER(ctypes.c_double)), ("nprods", ctypes.POINTER(ctypes.c_int)),
        ("c", ctypes.POINTER(ctypes.POINTER(ctypes.c_int))), ("method", ctypes.c_int),
        ("fixed", ctypes.c_int), ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
        ("device", ctypes.c_int),
    ]


class rdcu_info(ctypes.Structure):
    _fields_ = [
        ("state_len", ctypes.c_longlong), ("Y_len", ctypes.c_longlong),
        ("nnz_max", ctypes.c_longlong), ("n_channels", ctypes.c_int), ("order", ctypes.c_int),
        ("stream", ctypes.c_void_p), ("device_bytes", ctypes.c_longlong),
    ]


class rdcu_event(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("accepted", ctypes.c_int), ("steps", ctypes.c_int),
        ("eval_index", ctypes.c_int), ("order", ctypes.c_int), ("t", ctypes.c_double),
        ("h", ctypes.c_double), ("t_eval", ctypes.c_double), ("y", ctypes.c_void_p),
    ]


class rdcu_pass_timing(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("ms", ctypes.c_double), ("bytes", ctypes.c_double)]


OUT_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(rdcu_event))

_lib = None


def _addr(x) -> Optional[ctypes.c_void_p]:
    """A buffer argument as a C pointer.  Accepts an integer address (0 or None: NULL), a
    C-contiguous numpy array or a contiguous tensor (its ``data_ptr()``).  An array or
    tensor passed this way stays referenced for the whole call.  An address taken from
    a temporary (``np.array(y).ctypes.data``) does not: the library may read freed
    memory."""
    if x is None:
        return None
    if isinstance(x, numbers.Integral) and not isinstance(x, bool):
        return ctypes.c_void_p(int(x)) if int(x) else None
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_contiguous") and not x.is_contiguous():
            raise ValueError("tensor arguments must be contiguous")
        return ctypes.c_void_p(x.data_ptr())
    if hasattr(x, "__array_interface__") and hasattr(x, "flags"):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("array arguments must be C-contiguous")
        return ctypes.c_void_p(x.ctypes.data)
    raise TypeError("expected an address, a numpy array or a tensor, got %s" % type(x).__name__)


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Loads librdcu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("librdcu.so not found at %s; run `python -m rdcu_b200.build`" % p)
    lib = ctypes.CDLL(p)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    pd, pi = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.rdcu_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(rdcu_spec)]
    lib.rdcu_destroy.argtypes = [vp]
    lib.rdcu_set_state.argtypes = [vp, d, d, vp, i, vp]
    lib.rdcu_get_state.argtypes = [vp, pd, pd, pi, vp, vp]
    lib.rdcu_get_info.argtypes = [vp, ctypes.POINTER(rdcu_info)]
    lib.rdcu_rhs.argtypes = [vp, d, vp, vp, vp]
    lib.rdcu_jac.argtypes = [vp, d, vp, pi, vp, vp, vp]
    lib.rdcu_step.argtypes = [vp, pd, pd, d, d, pi]
    lib.rdcu_eval.argtypes = [vp, d, vp]
    lib.rdcu_solve.argtypes = [vp, d, d, d, pd, i, OUT_CB, vp]
    lib.rdcu_get_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    lib.rdcu_get_linear_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.POINTER(ctypes.c_longlong)]
    lib.rdcu_memcpy.argtypes = [vp, vp, vp, ctypes.c_ulonglong]
    lib.rdcu_advance.argtypes = [vp, i, d, d, ctypes.POINTER(ctypes.c_longlong)]
    lib.rdcu_random_ic.argtypes = [pd, i, ctypes.c_longlong, d, d, i]
    lib.rdcu_profile_passes.argtypes = [vp, i, ctypes.POINTER(rdcu_pass_timing), i, pi]
    lib.rdcu_rhs_noalloc.argtypes = [ctypes.POINTER(rdcu_spec), vp, vp, vp]
    lib.rdcu_set_coefficients.argtypes = [vp, pd]
    lib.rdcu_adjoint_forward.argtypes = [vp, vp, pd, i, i, vp]
    lib.rdcu_adjoint_backward.argtypes = [vp, vp, vp, pd]
    ll = ctypes.c_longlong
    lib.rdcu_ensemble_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(rdcu_spec), i]
    lib.rdcu_ensemble_destroy.argtypes = [vp]
    lib.rdcu_ensemble_set_state.argtypes = [vp, i, d, d, vp]
    lib.rdcu_ensemble_get_state.argtypes = [vp, i, pd, pd, vp]
    lib.rdcu_ensemble_solve.argtypes = [vp, d, d, d]
    lib.rdcu_ensemble_counters.argtypes = [vp, i, ctypes.POINTER(ll), ctypes.POINTER(ll)]
    lib.rdcu_ensemble_tune.argtypes = [vp, pi]
    lib.rdcu_ensemble_info.argtypes = [vp, pi, ctypes.POINTER(vp), ctypes.POINTER(ll)]
    lib.rdcu_ensemble_last_error.argtypes = [vp]
    lib.rdcu_ensemble_last_error.restype = ctypes.c_char_p
    pll = ctypes.POINTER(ll)
    lib.rdcu_lines_create.argtypes = [ctypes.POINTER(vp), pi, pd, i]
    lib.rdcu_lines_destroy.argtypes = [vp]
    lib.rdcu_lines_find.argtypes = [vp, vp, i, pll, pll, pll]
    lib.rdcu_lines_prefetch.argtypes = [vp, vp, i]
    lib.rdcu_lines_edges.argtypes = [vp, vp, vp]
    lib.rdcu_lines_cubes.argtypes = [vp, vp, vp]
    lib.rdcu_lines_correlate.argtypes = [vp, vp, vp]
    lib.rdcu_lines_correlate_sets.argtypes = [vp, vp, vp, ll, vp, vp, ll, vp]
    lib.rdcu_lines_profile.argtypes = [vp, vp, i, i, ctypes.POINTER(rdcu_pass_timing), i, pi]
    lib.rdcu_lines_info.argtypes = [vp, ctypes.POINTER(vp), pll, pll]
    lib.rdcu_lines_last_error.argtypes = [vp]
    lib.rdcu_lines_last_error.restype = ctypes.c_char_p
    lib.rdcu_error_string.argtypes = [i]
    lib.rdcu_error_string.restype = ctypes.c_char_p
    lib.rdcu_last_error.argtypes = [vp]
    lib.rdcu_last_error.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in _STRING_RESULTS:
            getattr(lib, name).restype = ctypes.c_int
    if path is None:
        _lib = lib
    return lib


def parse_terms(lines: Sequence[str]):
    """(C, ints) per coupling term from reference-format strings ``C,field,k,p,...``.
    The CLI (and the oracle) restate the reference's exact parser; this helper accepts
    well-formed terms only."""
    out = []
    for s in lines:
        toks = [t for t in s.split(",") if t != ""]
        out.append((float(toks[0]), [int(t) for t in toks[1:]]))
    return out


def random_ic(n: int, N: int, A: float, A0: float, seed: int):
    """The reference CLI's glibc-rand() initial condition (rdcu.cu:991-1001), as numpy."""
    import numpy as np

    lib = load_library()
    y = np.empty(n * N, np.float64)
    rc = lib.rdcu_random_ic(y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, N, A, A0, seed)
    if rc != RDCU_OK:
        raise RdcuError(rc, lib.rdcu_last_error(None).decode())
    return y


NOALLOC_SCRATCH_BYTES = 64 << 20


def rhs_noalloc(n: int, Ns: Sequence[int], Ls: Sequence[float], terms, y_ptr: Buffer, f_ptr: Buffer,
                stream: int = 0, device: int = 0) -> None:
    """f = RHS(y) of a pseudospectral problem through rdcu_rhs_noalloc, the entry point
    that allocates no device memory (for callers that cannot allocate: its scratch is a
    fixed 64 MiB device array inside the library).  y_ptr, f_ptr: device addresses of
    n*N doubles; stream: a cudaStream_t handle or 0."""
    lib = load_library()
    terms = [(float(C), list(ints)) for C, ints in terms]
    Cs = (ctypes.c_double * max(1, len(terms)))(*[t[0] for t in terms])
    nps = (ctypes.c_int * max(1, len(terms)))(*[len(t[1]) for t in terms])
    lists = [(ctypes.c_int * max(1, len(t[1])))(*t[1]) for t in terms]
    cps = (ctypes.POINTER(ctypes.c_int) * max(1, len(terms)))(
        *[ctypes.cast(l, ctypes.POINTER(ctypes.c_int)) for l in lists])
    spec = rdcu_spec()
    spec.n = n
    spec.ndim = len(Ns)
    for a in range(3):
        spec.Ns[a] = Ns[a] if a < len(Ns) else 1
        spec.Ls[a] = Ls[a] if a < len(Ns) else 1.0
    spec.nterms = len(terms)
    spec.C = ctypes.cast(Cs, ctypes.POINTER(ctypes.c_double))
    spec.nprods = ctypes.cast(nps, ctypes.POINTER(ctypes.c_int))
    spec.c = ctypes.cast(cps, ctypes.POINTER(ctypes.POINTER(ctypes.c_int)))
    spec.method = METHOD_DP45
    spec.device = device
    rc = lib.rdcu_rhs_noalloc(ctypes.byref(spec), _addr(y_ptr), _addr(f_ptr),
                              ctypes.c_void_p(stream) if stream else None)
    if rc != RDCU_OK:
        raise RdcuError(rc, lib.rdcu_last_error(None).decode())


class Solver:
    """One problem handle (``rdcu_t``)."""

    def __init__(self, n: int, Ns: Sequence[int], Ls: Sequence[float], terms, method: int = METHOD_DP45,
                 rtol: float = 1e-8, atol: float = 1e-8, fixed: bool = False, device: int = 0):
        self.lib = load_library()
        ndim = len(Ns)
        self.n, self.Ns, self.Ls = n, tuple(Ns), tuple(Ls)
        terms = [(float(C), list(ints)) for C, ints in terms]
        self._C = (ctypes.c_double * max(1, len(terms)))(*[t[0] for t in terms])
        self._np = (ctypes.c_int * max(1, len(terms)))(*[len(t[1]) for t in terms])
        self._lists = [(ctypes.c_int * max(1, len(t[1])))(*t[1]) for t in terms]
        self._c = (ctypes.POINTER(ctypes.c_int) * max(1, len(terms)))(
            *[ctypes.cast(l, ctypes.POINTER(ctypes.c_int)) for l in self._lists])
        spec = rdcu_spec()
        spec.n = n
        spec.ndim = ndim
        for a in range(3):
            spec.Ns[a] = Ns[a] if a < ndim else 1
            spec.Ls[a] = Ls[a] if a < ndim else 1.0
        spec.nterms = len(terms)
        spec.C = ctypes.cast(self._C, ctypes.POINTER(ctypes.c_double))
        spec.nprods = ctypes.cast(self._np, ctypes.POINTER(ctypes.c_int))
        spec.c = ctypes.cast(self._c, ctypes.POINTER(ctypes.POINTER(ctypes.c_int)))
        spec.method = method
        spec.fixed = 1 if fixed else 0
        spec.rtol = rtol
        spec.atol = atol
        spec.device = device
        h = ctypes.c_void_p()
        rc = self.lib.rdcu_create(ctypes.byref(h), ctypes.byref(spec))
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_last_error(None).decode())
        self.h = h
        self.method = method

    def _check(self, rc):
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.rdcu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> rdcu_info:
        inf = rdcu_info()
        self._check(self.lib.rdcu_get_info(self.h, ctypes.byref(inf)))
        return inf

    @property
    def stream(self) -> int:
        return self.info().stream

    def set_state(self, t: float, h: float, y_ptr: Buffer, order: int = 0, D_ptr: Buffer = 0):
        self._check(self.lib.rdcu_set_state(self.h, t, h, _addr(y_ptr), order, _addr(D_ptr)))

    def get_state(self, y_ptr: Buffer = 0, D_ptr: Buffer = 0):
        t, h, o = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.rdcu_get_state(self.h, ctypes.byref(t), ctypes.byref(h), ctypes.byref(o),
                                            _addr(y_ptr), _addr(D_ptr)))
        return t.value, h.value, o.value

    def rhs(self, y_ptr: Buffer, f_ptr: Buffer, Y_ptr: Buffer = 0, t: float = 0.0):
        self._check(self.lib.rdcu_rhs(self.h, t, _addr(y_ptr), _addr(f_ptr), _addr(Y_ptr)))

    def jac(self, y_ptr: Buffer, rows_ptr: Buffer, cols_ptr: Buffer, vals_ptr: Buffer, t: float = 0.0) -> int:
        nnz = ctypes.c_int()
        self._check(self.lib.rdcu_jac(self.h, t, _addr(y_ptr), ctypes.byref(nnz), _addr(rows_ptr),
                                      _addr(cols_ptr), _addr(vals_ptr)))
        return nnz.value

    def step(self, t: float, h: float, hmin: float = 0.0, hmax: float = float("inf")):
        tt, hh, acc = ctypes.c_double(t), ctypes.c_double(h), ctypes.c_int()
        self._check(self.lib.rdcu_step(self.h, ctypes.byref(tt), ctypes.byref(hh), hmin, hmax,
                                       ctypes.byref(acc)))
        return bool(acc.value), tt.value, hh.value

    def eval(self, t_eval: float, y_ptr: Buffer):
        self._check(self.lib.rdcu_eval(self.h, t_eval, _addr(y_ptr)))

    def solve(self, t1: float, t_eval: Sequence[float] = (), hmin: float = 0.0, hmax: float = float("inf"),
              callback: Optional[Callable[[rdcu_event], int]] = None):
        te = (ctypes.c_double * max(1, len(t_eval)))(*t_eval)

        def _cb(user, evp):
            try:
                return int(callback(evp.contents) or 0) if callback else 0
            except Exception:  # an exception in Python aborts the solve
                import traceback
                traceback.print_exc()
                return 1

        cb = OUT_CB(_cb)
        self._check(self.lib.rdcu_solve(self.h, t1, hmin, hmax, ctypes.cast(te, ctypes.POINTER(ctypes.c_double)),
                                        len(t_eval), cb, None))

    def memcpy(self, dst: Buffer, src: Buffer, nbytes: int):
        """Synchronous copy between host/device addresses."""
        self._check(self.lib.rdcu_memcpy(self.h, _addr(dst), _addr(src), nbytes))

    def copy_to_numpy(self, src: int, count: int):
        """float64 array of `count` values copied from a device address."""
        import numpy as np

        out = np.empty(count, np.float64)
        self.memcpy(out.ctypes.data, src, count * 8)
        return out

    def advance(self, n_attempts: int, hmin: float = 0.0, hmax: float = float("inf")) -> int:
        """Runs n attempts on the device; returns how many were accepted."""
        acc = ctypes.c_longlong()
        self._check(self.lib.rdcu_advance(self.h, n_attempts, hmin, hmax, ctypes.byref(acc)))
        return acc.value

    def profile_passes(self, reps: int = 20):
        """[(name, ms per launch, bytes per launch)] for each pass of DP45 stage 4, then
        stage 7's forward and inverse passes (rdcu_profile_passes)."""
        arr = (rdcu_pass_timing * 16)()
        npass = ctypes.c_int()
        self._check(self.lib.rdcu_profile_passes(self.h, reps, arr, 16, ctypes.byref(npass)))
        return [(arr[i].name.decode(), arr[i].ms, arr[i].bytes) for i in range(npass.value)]

    def counters(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.rdcu_get_counters(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def linear_stats(self):
        """BDF linear-solver statistics since creation: (GMRES iterations, linear solves,
        restart cycles); zeros for DP45 handles."""
        it, so, cy = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.rdcu_get_linear_stats(self.h, ctypes.byref(it), ctypes.byref(so), ctypes.byref(cy)))
        return it.value, so.value, cy.value

    @property
    def nterms(self) -> int:
        return len(self._lists)

    def set_coefficients(self, C: Sequence[float]):
        """New coefficient for every coupling term (same dictionary structure)."""
        if len(C) != self.nterms:
            raise ValueError("expected %d coefficients" % self.nterms)
        arr = (ctypes.c_double * max(1, len(C)))(*[float(c) for c in C])
        self._check(self.lib.rdcu_set_coefficients(self.h, arr))
        for k, c in enumerate(C):
            self._C[k] = float(c)

    def adjoint_forward(self, y0_ptr: Buffer, hs: Sequence[float], K: int = 50, yT_ptr: Buffer = 0):
        """DP45 over the step sizes hs from y0 (fixed steps), checkpointing every K steps."""
        arr = (ctypes.c_double * max(1, len(hs)))(*[float(h) for h in hs])
        self._check(self.lib.rdcu_adjoint_forward(self.h, _addr(y0_ptr), arr, len(hs), int(K), _addr(yT_ptr)))

    def adjoint_backward(self, lamT_ptr: Buffer, grad_y0_ptr: Buffer = 0):
        """dL/dy0 (written to grad_y0_ptr) and dL/dC (returned, one per term) of the last
        adjoint_forward, given dL/dyT at lamT_ptr."""
        g = (ctypes.c_double * max(1, self.nterms))()
        self._check(self.lib.rdcu_adjoint_backward(self.h, _addr(lamT_ptr), _addr(grad_y0_ptr), g))
        return [g[k] for k in range(self.nterms)]


class _SpecHolder:
    """An rdcu_spec with the term arrays it points to kept alive."""

    def __init__(self, n, Ns, Ls, terms, method=METHOD_DP45, rtol=1e-8, atol=1e-8, fixed=False, device=0):
        ndim = len(Ns)
        terms = [(float(C), list(ints)) for C, ints in terms]
        self._C = (ctypes.c_double * max(1, len(terms)))(*[t[0] for t in terms])
        self._np = (ctypes.c_int * max(1, len(terms)))(*[len(t[1]) for t in terms])
        self._lists = [(ctypes.c_int * max(1, len(t[1])))(*t[1]) for t in terms]
        self._c = (ctypes.POINTER(ctypes.c_int) * max(1, len(terms)))(
            *[ctypes.cast(l, ctypes.POINTER(ctypes.c_int)) for l in self._lists])
        sp = rdcu_spec()
        sp.n = n
        sp.ndim = ndim
        for a in range(3):
            sp.Ns[a] = Ns[a] if a < ndim else 1
            sp.Ls[a] = Ls[a] if a < ndim else 1.0
        sp.nterms = len(terms)
        sp.C = ctypes.cast(self._C, ctypes.POINTER(ctypes.c_double))
        sp.nprods = ctypes.cast(self._np, ctypes.POINTER(ctypes.c_int))
        sp.c = ctypes.cast(self._c, ctypes.POINTER(ctypes.POINTER(ctypes.c_int)))
        sp.method = method
        sp.fixed = 1 if fixed else 0
        sp.rtol = rtol
        sp.atol = atol
        sp.device = device
        self.spec = sp


class Ensemble:
    """Many 2D DP45 problems stepped together (``rdcu_ensemble_t``).

    ``members`` is a list of dicts with keys n, Ns, Ls, terms and optionally rtol, atol.
    """

    def __init__(self, members, device: int = 0):
        self.lib = load_library()
        holders = [_SpecHolder(m["n"], m["Ns"], m["Ls"], m["terms"], rtol=m.get("rtol", 1e-8),
                               atol=m.get("atol", 1e-8), device=device) for m in members]
        arr = (rdcu_spec * len(holders))(*[h.spec for h in holders])
        e = ctypes.c_void_p()
        rc = self.lib.rdcu_ensemble_create(ctypes.byref(e), arr, len(holders))
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_ensemble_last_error(None).decode())
        self.e = e
        self.sizes = [m["n"] * m["Ns"][0] * m["Ns"][1] for m in members]

    def _check(self, rc):
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_ensemble_last_error(self.e).decode())

    def close(self):
        if getattr(self, "e", None):
            self.lib.rdcu_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.sizes)

    def set_state(self, i: int, t: float, h: float, y_ptr: Buffer):
        self._check(self.lib.rdcu_ensemble_set_state(self.e, i, t, h, _addr(y_ptr)))

    def get_state(self, i: int, y_ptr: Buffer = 0):
        t, h = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.rdcu_ensemble_get_state(self.e, i, ctypes.byref(t), ctypes.byref(h),
                                                     _addr(y_ptr)))
        return t.value, h.value

    def solve(self, t1: float, hmin: float = 0.0, hmax: float = float("inf")):
        self._check(self.lib.rdcu_ensemble_solve(self.e, t1, hmin, hmax))

    def counters(self, i: int):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.rdcu_ensemble_counters(self.e, i, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def tune(self) -> int:
        v = ctypes.c_int()
        self._check(self.lib.rdcu_ensemble_tune(self.e, ctypes.byref(v)))
        return v.value

    @property
    def stream(self) -> int:
        c, st, b = ctypes.c_int(), ctypes.c_void_p(), ctypes.c_longlong()
        self._check(self.lib.rdcu_ensemble_info(self.e, ctypes.byref(c), ctypes.byref(st), ctypes.byref(b)))
        return st.value

    @property
    def device_bytes(self) -> int:
        c, st, b = ctypes.c_int(), ctypes.c_void_p(), ctypes.c_longlong()
        self._check(self.lib.rdcu_ensemble_info(self.e, ctypes.byref(c), ctypes.byref(st), ctypes.byref(b)))
        return b.value

