"""Coupling lists of standard problems, as FILEBASEcoupling.dat text.

The reference's notebooks write these lists for its examples (cgle.ipynb): one term per
line, "C,field,Yidx,pow,..." with Y index = block * n + field, block 0 the field itself,
1..ndim the first derivatives and ndim+1+i*ndim+j the second derivatives d_i d_j.
"""
from __future__ import annotations

from typing import List


def cgle_coupling_lines(ndim: int, b: float = 2.0, c: float = 0.8) -> List[str]:
    """Complex Ginzburg-Landau dA/dt = A + (1+ib) lap A - (1-ic)|A|^2 A with A = u0 + i u1
    (n = 2 fields), 4*ndim + 10 terms."""
    n = 2

    def dd(i, j):  # Y index of d_j d_j u_i
        return n + ndim * n + (j * ndim + j) * n + i

    fmt = lambda v: ("%f" % v)  # signed value; never prefix a '-' to it
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
    """2D Brusselator u_t = 1 - 4u + u^2 v + lap u, v_t = 3u - u^2 v + 8 lap v (9 terms)."""
    return ["1.0,0", "-4.0,0,0,1", "1.0,0,0,2,1,1", "1.0,0,6,1", "1.0,0,12,1",
            "3.0,1,0,1", "-1.0,1,0,2,1,1", "8.0,1,7,1", "8.0,1,13,1"]
