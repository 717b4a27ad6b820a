"""Oracle: problem definition, coupling parser, initial conditions and file formats.

Test infrastructure only (see ``oracle/__init__``).  Every function cites the reference
code it restates.
"""
from __future__ import annotations

import ctypes
import math
import re
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

# rdcu.cu:14
PI = 3.14159265358979323846
# glibc RAND_MAX (rdcu.cu:996 divides by it)
RAND_MAX = 2147483647

_FLOAT_RE = re.compile(
    r"^[ \t\n\r\f\v]*([+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))",
    re.IGNORECASE,
)
_INT_RE = re.compile(r"^[ \t\n\r\f\v]*([+-]?\d+)")


def c_atof(s: str) -> float:
    """C ``atof``: parse the longest numeric prefix, 0.0 if there is none."""
    m = _FLOAT_RE.match(s)
    return float(m.group(1)) if m else 0.0


def c_atoi(s: str) -> int:
    """C ``atoi``: parse the longest integer prefix, 0 if there is none."""
    m = _INT_RE.match(s)
    if not m:
        return 0
    v = int(m.group(1))
    # atoi returns an int; wrap like a 32-bit two's-complement conversion
    return ((v + 2**31) % 2**32) - 2**31


def _strtok(s: str, delim: str) -> List[Tuple[int, str]]:
    """Tokens of ``s`` split on any character of ``delim`` with empty tokens skipped,
    as ``strtok`` yields them, each with its start offset."""
    out = []
    i = 0
    n = len(s)
    while i < n:
        while i < n and s[i] in delim:
            i += 1
        if i >= n:
            break
        j = i
        while j < n and s[j] not in delim:
            j += 1
        out.append((i, s[i:j]))
        i = j
    return out


@dataclass
class Term:
    """One coupling term C * prod_k Y_k^eta, added to field ``field``.

    ``ints`` is the raw integer list that the reference stores in ``c[i]``
    (rdcu.cu:606,656-658): ``ints[0]`` is the field, then (Y index, power) pairs.
    """

    C: float
    ints: List[int]

    @property
    def field(self) -> int:
        # c[i][0]; c[i] is calloc'ed, so an empty list reads field 0 (rdcu.cu:656,832)
        return self.ints[0] if self.ints else 0

    @property
    def pairs(self) -> List[Tuple[int, int]]:
        """(Y index, power) pairs exactly as the loops at rdcu.cu:178-180 read them:
        j = 1, 3, ... < nprods, with c[i][j+1] read past the parsed list as 0 (calloc)."""
        out = []
        nprods = len(self.ints)
        for j in range(1, nprods, 2):
            k = self.ints[j]
            p = self.ints[j + 1] if j + 1 < nprods else 0
            out.append((k, p))
        return out


def parse_term(arg: str, delim: str = ",") -> Term | None:
    """One coupling term from a ``-c`` argument or a coupling-file token.

    Restates rdcu.cu:654-660 / 831-834: ``fparse_list`` (rdcu.cu:359-374) reads exactly
    one double (the coefficient) and reports ``strlen(token)+1`` characters consumed;
    ``parse_list`` (rdcu.cu:343-357) then reads the integers from that offset.
    Returns None when no coefficient token exists (the reference then indexes c[-1],
    which is undefined behaviour; the library rejects such input).
    """
    toks = _strtok(arg, delim)
    if not toks:
        return None
    C = c_atof(toks[0][1])
    chars = len(toks[0][1]) + 1
    rest = arg[chars:] if chars <= len(arg) else ""
    ints = [c_atoi(t) for _, t in _strtok(rest, delim)][:1024]
    return Term(C, ints)


def read_coupling_file(path: str) -> List[Term]:
    """Terms from ``FILEBASEcoupling.dat``: whitespace-separated tokens, one term per
    token (``fscanf(in, "%s", line)``, rdcu.cu:823-837)."""
    terms = []
    with open(path, "r") as fh:
        for tok in fh.read().split():
            t = parse_term(tok)
            if t is not None:
                terms.append(t)
    return terms


def y_names(n: int, ndim: int) -> List[str]:
    """Y-index table printed by ``-h`` (rdcu.cu:769-785) and used in the verbose
    equation print (rdcu.cu:789-805).  Index k = Yind*n + field."""
    names = [f"u{i}" for i in range(n)]
    for j in range(ndim):
        for i in range(n):
            names.append(f"u{i}_{j}")
    for j in range(ndim):
        for k in range(ndim):
            for i in range(n):
                names.append(f"u{i}_{j}{k}")
    return names


@dataclass
class Problem:
    """Problem context (restates the fields of ``parameters``, rdcu.cu:17-76, that the
    RHS reads)."""

    n: int
    Ns: Tuple[int, ...]
    Ls: Tuple[float, ...]
    terms: List[Term] = field(default_factory=list)

    @property
    def ndim(self) -> int:
        return len(self.Ns)

    @property
    def N(self) -> int:
        return int(np.prod(self.Ns))

    @property
    def nY(self) -> int:
        """Number of Y blocks per field: 1 + ndim + ndim^2 (rdcu.cu:900)."""
        return 1 + self.ndim + self.ndim * self.ndim


def glibc_uniform_ic(n: int, N: int, A: float, A0: float, seed: int) -> np.ndarray:
    """Random initial condition of rdcu.cu:898,994-1001:
    ``srand(seed)``; ``y[N*i+j] = A0 + A/2*(2.0/RAND_MAX*rand()-1)`` with the field loop
    outer.  Uses the C library's own ``srand``/``rand`` so the stream is identical."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed & 0xFFFFFFFF))
    y = np.empty(n * N, dtype=np.float64)
    half_a = A / 2
    scale = 2.0 / RAND_MAX
    for idx in range(n * N):
        r = libc.rand()
        y[idx] = A0 + half_a * (scale * r - 1)
    return y


def t_eval_grid(t: float, t1: float, dt: float) -> np.ndarray:
    """Output times of rdcu.cu:1052-1059: dt*k for k = int(t/dt)+1 ... int(t1/dt)."""
    n0 = int(t / dt) + 1
    n1 = int(t1 / dt) + 1
    return np.array([dt * nn for nn in range(n0, n1)], dtype=np.float64)


# ----------------------------------------------------------------------------- formats
def write_fs(path: str, y: np.ndarray, t: float, h: float, order: int | None = None,
             D: Sequence[np.ndarray] | None = None) -> None:
    """``FILEBASEfs.dat`` (rdcu.cu:320-339): y (n*N f64), t, h; BDF adds int32 order and
    D_1..D_order (order*n*N f64)."""
    with open(path, "wb") as fh:
        fh.write(np.asarray(y, np.float64).tobytes())
        fh.write(np.float64(t).tobytes())
        fh.write(np.float64(h).tobytes())
        if order is not None:
            fh.write(np.int32(order).tobytes())
            for i in range(1, order + 1):
                fh.write(np.asarray(D[i], np.float64).tobytes())


def read_fs(path: str, nN: int, stiff: bool):
    """Reads ``fs.dat`` as rdcu.cu:944-990 does; returns (y, t, h, order, D list)."""
    raw = open(path, "rb").read()
    y = np.frombuffer(raw, np.float64, nN, 0).copy()
    off = nN * 8
    t, h = np.frombuffer(raw, np.float64, 2, off)
    off += 16
    order, D = 0, []
    if stiff and len(raw) >= off + 4:
        order = int(np.frombuffer(raw, np.int32, 1, off)[0])
        off += 4
        for i in range(order):
            D.append(np.frombuffer(raw, np.float64, nN, off).copy())
            off += nN * 8
    return y, float(t), float(h), order, D


def pow_c(x: np.ndarray, eta: float) -> np.ndarray:
    """``pow(double, double)`` elementwise with C semantics for the integer exponents the
    dictionary uses (pow(x, 0) == 1 for every x, including NaN)."""
    with np.errstate(all="ignore"):
        return np.power(x, float(eta))


def isclose_rel(a: np.ndarray, b: np.ndarray) -> float:
    """Max-norm relative difference |a-b|_inf / max(|b|_inf, tiny)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b))) / den if a.size else 0.0


def cgle_terms(ndim: int, b: float = 2.0, c: float = 0.8) -> List[Term]:
    """The CGLE coupling terms of :func:`cgle_coupling_lines`, parsed."""
    return [parse_term(s) for s in cgle_coupling_lines(ndim, b, c)]


def cgle_coupling_lines(ndim: int, b: float = 2.0, c: float = 0.8) -> List[str]:
    """The CGLE coupling list the reference notebook writes to ``coupling.dat``
    (cgle.ipynb cell 3 for 2D, cell 31 for 3D), for any ndim: A = u0 + i u1,
    dA/dt = A + (1+ib) lap A - (1-ic)|A|^2 A with n = 2 fields."""
    n = 2

    def dd(i, j):
        return n + ndim * n + (j * ndim + j) * n + i

    fmt = lambda v: ("%f" % v)  # signed: "-%s" % fmt(-2.0) would read "--2.0", which atof takes as 0
    lines = ["1.0,0,0,1"]
    lines += ["1.0,0,%d,1" % dd(0, j) for j in range(ndim)]
    lines += ["%s,0,%d,1" % (fmt(-b), dd(1, j)) for j in range(ndim)]
    lines += ["-1.0,0,0,3", "-1.0,0,0,1,1,2", "1.0,1,1,1"]
    lines += ["1.0,1,%d,1" % dd(1, j) for j in range(ndim)]
    lines += ["%s,1,%d,1" % (fmt(b), dd(0, j)) for j in range(ndim)]
    lines += ["-1.0,1,0,2,1,1", "-1.0,1,1,3", "%s,1,0,3" % fmt(c), "%s,1,0,1,1,2" % fmt(c),
              "%s,0,0,2,1,1" % fmt(-c), "%s,0,1,3" % fmt(-c)]
    return lines


def brusselator_coupling_lines() -> List[str]:
    """2D Brusselator u_t = 1 - 4u + u^2 v + lap u, v_t = 3u - u^2 v + 8 lap v as a
    9-term coupling list (n=2, ndim=2: u0_00 = 6, u0_11 = 12, u1_00 = 7, u1_11 = 13)."""
    return ["1.0,0", "-4.0,0,0,1", "1.0,0,0,2,1,1", "1.0,0,6,1", "1.0,0,12,1",
            "3.0,1,0,1", "-1.0,1,0,2,1,1", "8.0,1,7,1", "8.0,1,13,1"]
