"""Oracle: defect-line extraction from a 3D complex field -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy/scipy, the reference's post-processing of CGLE states
(``makelines.py``):

* ``winding``   -- the plaquette phase winding ``wloop`` (makelines.py:19-24);
* ``findlines`` -- line cubes, the face-neighbour graph and its connected components,
  returned as per-component edge lists of scaled cube coordinates (makelines.py:26-57,
  the numpy twin at :72-99);
* ``correlate`` -- the minimum periodic L1 distance between the cubes of every pair of
  components of consecutive frames (makelines.py:112-144, numpy twin :146-178);
* ``phase``     -- ``atan2(v, u) + pi`` of a stored state (makelines.py:65).

The reference builds the neighbour graph by an all-pairs distance test over the line
cubes and numbers components with networkx; this restatement builds the same graph
from the grid (periodic face neighbours) and labels it with scipy's connected
components.  Components come in networkx's order (by their smallest cube).  Within a
component the reference's edge order and orientation follow CPython set iteration
(networkx's subgraph views iterate the component's node set); this restatement gives
each edge as (u, v), u < v, in lexicographic order of the cubes' C-order indices, and
the parity tests compare edge sets in that canonical form (every consumer of the
edges in the reference -- correlate's ``np.unique``, the ancestry's edge counts -- is
order-free).  Pinned to the reference's own functions by the fixtures under
``tests/golden`` (``make_lines_golden.py``).

Only ``tests/`` and ``bench.py`` may import it (see ``oracle/__init__``).
"""
from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components

TWO_PI = 2 * np.pi


def phase(y: np.ndarray, Ns) -> np.ndarray:
    """Phase of a 2-field state (u block then v block) as makelines.py:65 forms it."""
    ys = np.asarray(y, dtype=np.float64).reshape((2,) + tuple(int(n) for n in Ns))
    return np.arctan2(ys[1], ys[0]) + np.pi


def _wrap(x: np.ndarray) -> np.ndarray:
    """Phase difference mapped to [-pi, pi): numpy's floored float modulus."""
    return np.mod(x + np.pi, TWO_PI) - np.pi


def winding(th: np.ndarray, a: int, b: int) -> np.ndarray:
    """Winding number of the plaquette at every point spanned by axis a, then axis b
    (makelines.py:19-24): the four wrapped differences around p, p+e_a, p+e_a+e_b,
    p+e_b, summed in that order, over 2*pi, rounded."""
    t1 = np.roll(th, -1, axis=a)
    t2 = np.roll(t1, -1, axis=b)
    t3 = np.roll(th, -1, axis=b)
    s = _wrap(t1 - th) + _wrap(t2 - t1) + _wrap(t3 - t2) + _wrap(th - t3)
    return np.round(s / TWO_PI)


def line_cubes(th: np.ndarray) -> np.ndarray:
    """Boolean mask of the cubes a defect line passes through: the two cubes on either
    side of every plaquette with nonzero winding (makelines.py:28-36).  A plaquette of
    the (0,1) plane at p borders cubes p and p - e2; of the (1,2) plane, p and p - e0;
    of the (2,0) plane, p and p - e1."""
    w01 = winding(th, 0, 1) != 0
    w12 = winding(th, 1, 2) != 0
    w20 = winding(th, 2, 0) != 0
    return (w01 | np.roll(w01, -1, axis=2) | w12 | np.roll(w12, -1, axis=0) | w20 |
            np.roll(w20, -1, axis=1))


def neighbour_pairs(cubes: np.ndarray, Ns) -> tuple[np.ndarray, np.ndarray]:
    """All (u, v), u < v, of marked cubes at periodic L1 distance 1 (makelines.py:41-50:
    per-axis difference mapped to [-N/2, N/2) by (d + N//2) mod N - N//2), as indices
    into the sorted cube list."""
    Ns = tuple(int(n) for n in Ns)
    N = int(np.prod(Ns))
    rank = np.full(N, -1, dtype=np.int64)
    rank[cubes] = np.arange(cubes.size)
    coords = np.array(np.unravel_index(cubes, Ns))
    us, vs = [], []
    for axis in range(3):
        if Ns[axis] < 2:
            continue
        for step in (1, -1):
            c = coords.copy()
            c[axis] = (c[axis] + step) % Ns[axis]
            nb = rank[np.ravel_multi_index(c, Ns)]
            ok = nb > np.arange(cubes.size)
            us.append(np.nonzero(ok)[0])
            vs.append(nb[ok])
    u = np.concatenate(us) if us else np.zeros(0, np.int64)
    v = np.concatenate(vs) if vs else np.zeros(0, np.int64)
    key = np.unique(u * max(cubes.size, 1) + v)  # sorted, duplicates (N = 2) merged
    return key // max(cubes.size, 1), key % max(cubes.size, 1)


def components(cubes: np.ndarray, Ns):
    """Per-cube component index (components numbered by their smallest cube) and the
    sorted neighbour pairs."""
    u, v = neighbour_pairs(cubes, Ns)
    n = cubes.size
    g = coo_matrix((np.ones(u.size), (u, v)), shape=(n, n))
    _, lab = connected_components(g, directed=False)
    first = np.full(lab.max() + 1 if n else 0, n, dtype=np.int64)
    np.minimum.at(first, lab, np.arange(n))
    order = np.argsort(first, kind="stable")
    remap = np.empty_like(order)
    remap[order] = np.arange(order.size)
    return remap[lab] if n else lab, u, v


def findlines(th: np.ndarray, Ns, Ls) -> list[np.ndarray]:
    """Per component (ordered by smallest cube), its edges as an array (E, 2, 3) of cube
    coordinates c scaled as (c * Ls) / (Ns - 1) (makelines.py:55-56).  A field without
    lines gives [] (the reference raises ValueError there)."""
    Ns = np.asarray(Ns)
    Ls = np.asarray(Ls, dtype=np.float64)
    cubes = np.nonzero(line_cubes(np.asarray(th, dtype=np.float64)).ravel())[0]
    if cubes.size == 0:
        return []
    comp, u, v = components(cubes, Ns)
    coords = np.array(np.unravel_index(cubes, tuple(int(n) for n in Ns)))  # (3, n)
    out = []
    ec = comp[u]
    for c in range(comp.max() + 1):
        sel = ec == c
        e = np.stack([coords[:, u[sel]], coords[:, v[sel]]], axis=0)  # (2, 3, E)
        out.append(e.transpose(2, 0, 1) * Ls / (Ns - 1))  # (c * L) / (N - 1), in that order
    return out


def canonical(edges: np.ndarray, Ns, Ls) -> np.ndarray:
    """A component's edges (E, 2, 3) as cube-index pairs (u, v), u < v, sorted: the
    form in which edge lists are compared (the cube coordinate is recovered by
    rounding x * (N - 1) / L)."""
    Ns = np.asarray(Ns)
    q = np.round(np.asarray(edges) * (Ns - 1) / np.asarray(Ls, dtype=np.float64)).astype(np.int64)
    idx = np.ravel_multi_index(q.reshape(-1, 3).T, tuple(int(n) for n in Ns)).reshape(-1, 2)
    idx = np.sort(idx, axis=1)
    return idx[np.lexsort((idx[:, 1], idx[:, 0]))]


def _cube_sets(frame, Ns, Ls, truncate):
    s = np.asarray(Ls, dtype=np.float64) / (np.asarray(Ns) - 1)
    sets = []
    for comp in frame:
        x = np.concatenate(comp / s, axis=0)  # (2E, 3)
        q = x.astype(int) if truncate else np.round(x).astype(int)
        sets.append(np.unique(np.ravel_multi_index(q.T, tuple(int(n) for n in Ns))))
    return sets


def correlate(prev, cur, Ns, Ls) -> np.ndarray:
    """diffs[j, i]: minimum periodic L1 distance between the cubes of component i of
    the previous frame and component j of the current one (makelines.py:112-144).  The
    previous frame's coordinates are rounded back to cubes, the current frame's
    truncated, as the reference does."""
    Ns = tuple(int(n) for n in Ns)
    a = _cube_sets(prev, Ns, Ls, False)
    b = _cube_sets(cur, Ns, Ls, True)
    out = np.zeros((len(b), len(a)), dtype=np.int64)
    half = np.array([n // 2 for n in Ns])[:, None, None]
    Nv = np.array(Ns)[:, None, None]
    for i, sa in enumerate(a):
        ca = np.array(np.unravel_index(sa, Ns))
        for j, sb in enumerate(b):
            cb = np.array(np.unravel_index(sb, Ns))
            d = np.mod(ca[:, :, None] - cb[:, None, :] + half, Nv) - half
            out[j, i] = np.abs(d).sum(axis=0).min()
    return out
