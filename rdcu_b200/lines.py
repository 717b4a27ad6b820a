"""Defect lines of 3D CGLE states on the GPU: the reference's makelines.py functions.

The reference tracks the phase defects ("vortex lines") of 3D complex Ginzburg-Landau
states in Python (makelines.py).  This module keeps its functions and arguments and
runs the per-frame work through ``rdcu_lines_*`` of librdcu:

* ``findlines(th, Ns, Ls, chunk, device)`` -- per connected component of line cubes,
  its edges as an (E, 2, 3) array of cube coordinates scaled (c * L) / (N - 1)
  (makelines.py:26-57);
* ``savelines(n, filename, Ns, Ls, n0, chunk, device)`` -- the same for frame n0 + n of
  a ``states.dat`` file (makelines.py:59-68), with the phase formed on the GPU;
* ``correlate(n, lines, Ns, Ls, chunk, device)`` -- minimum periodic L1 distances
  between the components of frames n - 1 and n (makelines.py:112-144);
* ``loadfaces(n, filebase, Ns, n0)`` -- the six boundary faces of a frame
  (makelines.py:180-186);
* ``ancestry(lines, results, thr)`` -- line ids, colour ids and parent edges, the
  reference's ``__main__`` ancestry block (makelines.py:322-387).

``Lines`` is the handle behind them: it keeps the last frame's results on the device,
so a frame sequence is found and correlated without leaving the GPU.

Differences from the reference: a frame without lines gives ``[]`` (the reference
raises ValueError); within a component the edges come as (u, v), u < v, in ascending
C-order of the cubes, where the reference's order follows Python set iteration inside
networkx -- the components, their order and every edge are the same.  ``chunk`` only
sized the reference's all-pairs blocks and is ignored; ``device`` must name a CUDA
device (there is no CPU path).
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import numpy as np

from . import RDCU_OK, RdcuError, load_library

STATE = 0  # RDCU_LINES_STATE: u block then v block
PHASE = 1  # RDCU_LINES_PHASE: theta = atan2(v, u) + pi


def _device_index(device) -> int:
    if device is None:
        return 0
    if isinstance(device, int):
        return device
    d = str(device)
    if d == "cuda":
        return 0
    if d.startswith("cuda:"):
        return int(d[5:])
    raise ValueError("defect-line extraction runs on a CUDA device, not %r" % (device,))


def _ptr(a) -> Tuple[int, object]:
    """(address, keep-alive) of a float64 numpy array, a CUDA/pinned torch tensor or an
    int address."""
    if isinstance(a, int):
        return a, None
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr()), a
    arr = np.ascontiguousarray(a, dtype=np.float64)
    return arr.ctypes.data, arr


class Lines:
    """Defect-line workspace for one 3D grid (``rdcu_lines_t``)."""

    def __init__(self, Ns: Sequence[int], Ls: Sequence[float], device: int = 0):
        self.lib = load_library()
        self.Ns = tuple(int(n) for n in Ns)
        self.Ls = tuple(float(x) for x in Ls)
        if len(self.Ns) != 3 or len(self.Ls) != 3:
            raise ValueError("defect lines need a 3D grid")
        h = ctypes.c_void_p()
        rc = self.lib.rdcu_lines_create(ctypes.byref(h), (ctypes.c_int * 3)(*self.Ns),
                                        (ctypes.c_double * 3)(*self.Ls), int(device))
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_lines_last_error(None).decode())
        self.h = h
        self.N = int(np.prod(self.Ns))
        self.counts = (0, 0, 0)
        self._staged = None

    def _check(self, rc):
        if rc != RDCU_OK:
            raise RdcuError(rc, self.lib.rdcu_lines_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.rdcu_lines_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_len(self, src, kind):
        need = (2 if kind == STATE else 1) * self.N
        if not isinstance(src, int) and int(np.prod(getattr(src, "shape", (len(src),)))) != need:
            raise ValueError("source must hold %d values" % need)

    def prefetch(self, src, kind: int = STATE) -> None:
        """Starts copying a host frame (pinned, e.g. a pinned torch tensor, for the copy to
        overlap) into the staging buffer; ``find(None, kind)`` uses it.  The last frame's
        results stay valid meanwhile."""
        self._check_len(src, kind)
        p, keep = _ptr(src)
        self._check(self.lib.rdcu_lines_prefetch(self.h, ctypes.c_void_p(p), kind))
        self._staged = keep  # the source must outlive the asynchronous copy

    def find(self, src, kind: int = STATE) -> Tuple[int, int, int]:
        """One frame: ``src`` is a state (2*N doubles, ``kind=STATE``) or a phase field
        (N doubles, ``kind=PHASE``) -- a numpy array, a torch tensor (CUDA or host) or a
        raw address -- or None for the frame staged by ``prefetch``.  Returns (line
        cubes, edges, components)."""
        if src is None:  # the frame staged by prefetch
            p, keep = 0, None
        else:
            self._check_len(src, kind)
            p, keep = _ptr(src)
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.rdcu_lines_find(self.h, ctypes.c_void_p(p), kind, ctypes.byref(a), ctypes.byref(b),
                                             ctypes.byref(c)))
        del keep
        self._staged = None
        self.counts = (a.value, b.value, c.value)
        return self.counts

    def edges(self) -> Tuple[np.ndarray, np.ndarray]:
        """(xyz of shape (E, 2, 3), component offsets into it) of the last frame."""
        _, ne, nc = self.counts
        xyz = np.empty((ne, 2, 3), dtype=np.float64)
        off = np.empty(nc + 1, dtype=np.int64)
        self._check(self.lib.rdcu_lines_edges(self.h, ctypes.c_void_p(xyz.ctypes.data if ne else 0),
                                              ctypes.c_void_p(off.ctypes.data)))
        return xyz, off

    def lines(self) -> List[np.ndarray]:
        """The last frame in the reference's form: one (E, 2, 3) array per component."""
        xyz, off = self.edges()
        return [xyz[off[c]:off[c + 1]] for c in range(len(off) - 1)]

    def cubes(self) -> Tuple[np.ndarray, np.ndarray]:
        """(C-order cube indices grouped by component, component offsets)."""
        n, _, nc = self.counts
        idx = np.empty(n, dtype=np.int64)
        off = np.empty(nc + 1, dtype=np.int64)
        self._check(self.lib.rdcu_lines_cubes(self.h, ctypes.c_void_p(idx.ctypes.data if n else 0),
                                              ctypes.c_void_p(off.ctypes.data)))
        return idx, off

    def correlate(self, prev: "Lines") -> np.ndarray:
        """diffs[j, i] between component i of ``prev``'s last frame and component j of
        this handle's last frame (makelines.py:112-144)."""
        out = np.empty((self.counts[2], prev.counts[2]), dtype=np.int64)
        self._check(self.lib.rdcu_lines_correlate(prev.h, self.h, ctypes.c_void_p(out.ctypes.data if out.size else 0)))
        return out

    def correlate_sets(self, prev_sets: Sequence[np.ndarray], cur_sets: Sequence[np.ndarray]) -> np.ndarray:
        """diffs[j, i] between explicit cube sets (C-order indices per component)."""
        def pack(sets):
            off = np.zeros(len(sets) + 1, dtype=np.int64)
            off[1:] = np.cumsum([len(s) for s in sets])
            cat = np.ascontiguousarray(np.concatenate(sets) if len(sets) else np.zeros(0), dtype=np.int64)
            return cat, off

        a, ao = pack(prev_sets)
        b, bo = pack(cur_sets)
        out = np.empty((len(cur_sets), len(prev_sets)), dtype=np.int64)
        self._check(self.lib.rdcu_lines_correlate_sets(
            self.h, ctypes.c_void_p(a.ctypes.data if a.size else 0), ctypes.c_void_p(ao.ctypes.data), len(prev_sets),
            ctypes.c_void_p(b.ctypes.data if b.size else 0), ctypes.c_void_p(bo.ctypes.data), len(cur_sets),
            ctypes.c_void_p(out.ctypes.data if out.size else 0)))
        return out

    def profile(self, src, kind: int = STATE, reps: int = 5) -> List[Tuple[str, float, float]]:
        """(pass, mean ms, algorithmic bytes) of each pass group of one find on ``src``.
        The handle keeps that frame (its counts are refreshed here, since ``edges`` and
        ``cubes`` size their arrays from them)."""
        from . import rdcu_pass_timing

        self.find(src, kind)
        p, keep = _ptr(src)
        arr = (rdcu_pass_timing * 16)()
        n = ctypes.c_int()
        self._check(self.lib.rdcu_lines_profile(self.h, ctypes.c_void_p(p), kind, reps, arr, 16, ctypes.byref(n)))
        del keep
        return [(arr[i].name.decode(), arr[i].ms, arr[i].bytes) for i in range(n.value)]

    def info(self) -> Tuple[int, int, int]:
        """(stream address, device bytes, kernels launched so far)."""
        st, b, k = ctypes.c_void_p(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.rdcu_lines_info(self.h, ctypes.byref(st), ctypes.byref(b), ctypes.byref(k)))
        return st.value or 0, b.value, k.value

    @property
    def stream(self) -> int:
        return self.info()[0]


_handles = {}


def _handle(Ns, Ls, device) -> Lines:
    key = (tuple(int(n) for n in Ns), tuple(float(x) for x in Ls), _device_index(device))
    h = _handles.get(key)
    if h is None:
        h = _handles[key] = Lines(key[0], key[1], key[2])
    return h


def findlines(th, Ns, Ls, chunk: int = 1024, device="cuda") -> List[np.ndarray]:
    """Line components of the phase field ``th`` (makelines.py:26-57)."""
    h = _handle(Ns, Ls, device)
    h.find(th if hasattr(th, "data_ptr") else np.asarray(th, dtype=np.float64).reshape(-1), PHASE)
    return h.lines()


def read_frame(filename: str, Ns, index: int) -> np.ndarray:
    """Frame ``index`` of a states.dat file: 2*N doubles (makelines.py:60-64)."""
    N = int(np.prod(Ns))
    return np.fromfile(filename, dtype=np.float64, count=2 * N, offset=index * 8 * 2 * N)


def savelines(n, filename, Ns, Ls, n0, chunk: int = 1024, device="cuda") -> List[np.ndarray]:
    """Line components of frame n0 + n of ``filename`` (makelines.py:59-68)."""
    h = _handle(Ns, Ls, device)
    h.find(read_frame(filename, Ns, n0 + n), STATE)
    return h.lines()


def _cube_sets(frame, Ns, Ls, truncate: bool) -> List[np.ndarray]:
    # cube coordinates recovered from the scaled edge coordinates: rounded for the earlier
    # frame, truncated for the later one (makelines.py:115,120)
    s = np.asarray(Ls, dtype=np.float64) / (np.asarray(Ns) - 1)
    out = []
    for comp in frame:
        x = np.concatenate(comp / s, axis=0) if len(comp) else np.zeros((0, 3))
        q = x.astype(int) if truncate else np.round(x).astype(int)
        out.append(np.unique(np.ravel_multi_index(q.T, tuple(int(v) for v in Ns))))
    return out


def correlate(n, lines, Ns, Ls, chunk: int = 1024, device="cuda") -> np.ndarray:
    """diffs[j, i]: minimum periodic L1 distance between component i of lines[n - 1] and
    component j of lines[n] (makelines.py:112-144)."""
    h = _handle(Ns, Ls, device)
    return h.correlate_sets(_cube_sets(lines[n - 1], Ns, Ls, False), _cube_sets(lines[n], Ns, Ls, True))


def loadfaces(n, filebase, Ns, n0) -> list:
    """The six boundary faces (u and v) of frame n0 + n of ``filebase``states.dat
    (makelines.py:180-186)."""
    ys = read_frame(filebase + "states.dat", Ns, n0 + n).reshape((2,) + tuple(int(v) for v in Ns))
    return [ys[:, 0, :, :], ys[:, :, 0, :], ys[:, :, :, 0], ys[:, -1, :, :], ys[:, :, -1, :], ys[:, :, :, -1]]


def ancestry(lines, results, thr: int):
    """Line ids, colour ids and ancestry edges of a frame sequence (makelines.py:322-387).

    ``lines[n]`` is frame n's component list (only the edge counts are used) and
    ``results[n]`` the correlate matrix of frames n and n + 1.  A component's parents are
    the previous frame's components at the row minimum, if that minimum is <= thr;
    components with the same parent list are siblings (components without parents are
    all siblings of one another).  A component keeps its parent's id only when it has
    exactly one parent and no sibling; otherwise it gets a new id, and its colour comes
    from the longest parent if it is the longest of its siblings (first maximum), else a
    new colour.  Every parent -> child id pair with a new id is an ancestry edge."""
    lengths = [[len(c) for c in frame] for frame in lines]
    nt = len(lines)
    parents = [[[i] for i in range(len(lines[0]))]]
    for n in range(nt - 1):
        r = np.asarray(results[n])
        ps = []
        for i in range(r.shape[0]):
            row = r[i]
            m = row.min() if row.size else None
            ps.append(np.nonzero(row == m)[0].tolist() if m is not None and m <= thr else [])
        parents.append(ps)
    siblings = []
    for ps in parents:
        groups = {}
        for m, p in enumerate(ps):
            groups.setdefault(tuple(p), []).append(m)
        siblings.append([groups[tuple(p)] for p in ps])
    ids = [np.arange(len(lines[0]))]
    cids = [np.arange(len(lines[0]))]
    nextid = nextcid = len(lines[0])
    edges = []
    for n in range(1, nt):
        k = len(parents[n])
        i_n = np.zeros(k, dtype=int)
        c_n = np.zeros(k, dtype=int)
        for m in range(k):
            ps, sb = parents[n][m], siblings[n][m]
            if len(ps) == 1 and len(sb) == 1:
                i_n[m] = ids[n - 1][ps[0]]
                c_n[m] = cids[n - 1][ps[0]]
                continue
            i_n[m] = nextid
            nextid += 1
            if not ps:
                c_n[m] = nextcid
                nextcid += 1
            else:
                longest_parent = ps[int(np.argmax(np.asarray(lengths[n - 1])[ps]))]
                longest_sibling = sb[int(np.argmax(np.asarray(lengths[n])[sb]))]
                if m == longest_sibling:
                    c_n[m] = cids[n - 1][longest_parent]
                else:
                    c_n[m] = nextcid
                    nextcid += 1
            for p in ps:
                edges.append([ids[n - 1][p], i_n[m]])
        ids.append(i_n)
        cids.append(c_n)
    return ids, cids, edges
