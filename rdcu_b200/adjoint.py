"""Discrete adjoint of DP45 as a ``torch.autograd.Function``.

``integrate(solver, y0, C, hs, K)`` maps the initial state ``y0`` (float64 CUDA tensor
of n*N values, fields outermost like the reference's state vector) and the coupling
coefficients ``C`` (one per term of the coupling file) to the state after the steps
``hs`` of fixed-step Dormand-Prince 4(5) (dp45.cu:34-69 with the b row of dp45.cu:11).
Its backward pass is the discrete adjoint in ``librdcu`` (``rdcu_adjoint_backward``):
checkpoints every K steps, stage states recomputed per segment, transposed spectral
derivative operators and monomial product rules in hand-written kernels.

The reference has no gradients; this module is the differentiable front end of the
same solver.  ``solver`` must be a pseudospectral ``rdcu_b200.Solver`` created with
``fixed=True``.
"""
from __future__ import annotations

from typing import Sequence

import torch

from . import Solver


def _sync():
    torch.cuda.current_stream().synchronize()


class DP45Adjoint(torch.autograd.Function):
    """yT = Phi_hs(y0; C).  Gradients flow to y0 and C."""

    @staticmethod
    def forward(ctx, y0: torch.Tensor, C: torch.Tensor, solver: Solver, hs: Sequence[float], K: int):
        if y0.dtype != torch.float64 or not y0.is_cuda:
            raise TypeError("y0 must be a float64 CUDA tensor")
        y0c = y0.detach().contiguous()
        Cl = [float(c) for c in C.detach().cpu().tolist()]
        _sync()
        solver.set_coefficients(Cl)
        yT = torch.empty_like(y0c)
        solver.adjoint_forward(y0c.data_ptr(), hs, K, yT.data_ptr())
        rec = object()
        solver._adjoint_record = rec
        ctx.solver, ctx.hs, ctx.K, ctx.Cl, ctx.rec = solver, list(hs), K, Cl, rec
        ctx.C_device, ctx.C_dtype = C.device, C.dtype
        ctx.save_for_backward(y0c)
        return yT

    @staticmethod
    def backward(ctx, gT: torch.Tensor):
        (y0c,) = ctx.saved_tensors
        s = ctx.solver
        _sync()
        if getattr(s, "_adjoint_record", None) is not ctx.rec:
            # the checkpoints belong to another forward call: record this one again
            s.set_coefficients(ctx.Cl)
            s.adjoint_forward(y0c.data_ptr(), ctx.hs, ctx.K, 0)
            s._adjoint_record = ctx.rec
        lam = gT.detach().to(torch.float64).contiguous()
        gy0 = torch.empty_like(y0c)
        gC = s.adjoint_backward(lam.data_ptr(), gy0.data_ptr())
        gCt = torch.tensor(gC, dtype=ctx.C_dtype, device=ctx.C_device)
        return gy0, gCt, None, None, None


def integrate(solver: Solver, y0: torch.Tensor, C: torch.Tensor, hs: Sequence[float], K: int = 50) -> torch.Tensor:
    """Differentiable fixed-step DP45 over the step sizes ``hs`` (see module docstring)."""
    return DP45Adjoint.apply(y0, C, solver, list(hs), int(K))


def accepted_steps(solver: Solver, y0_ptr: int, t0: float, h0: float, t1: float, hmin: float = 0.0):
    """Step sizes of the accepted steps of an adaptive run from t0 to t1, for replaying
    the same sequence through ``integrate`` (the adjoint treats them as constants)."""
    from . import EV_ATTEMPT

    solver.set_state(t0, h0, y0_ptr)
    hs = []
    cur = [h0]  # the step size an attempt uses is the one the previous attempt proposed

    def cb(ev):
        if ev.kind == EV_ATTEMPT:
            if ev.accepted:
                hs.append(cur[0])
            cur[0] = ev.h
        return 0

    solver.solve(t1, (), hmin=hmin, callback=cb)
    return hs
