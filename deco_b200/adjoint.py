"""Differentiable CPR-GMRES solve: x = A(values)^{-1} b as a torch.autograd.Function.

Forward: CPR(prec, A, b) + SOL(sol, ...) on the device (the matrix and the
right-hand side are copied, the caller's tensors are not decoupled).  Only the
input values and the solution x are kept for the backward pass; the Krylov basis
is not stored.

Backward, for g = dL/dx:  A^T lam = g with CPR built on A^T (transposed, then
decoupled: deco_adjoint_create / deco_adjoint_solve), then
    dL/db = lam,    dL/dA_ij = -lam_i x_j on A's pattern (deco_grad_A_pattern).

Every step runs in libdeco_b200.so; there is no CPU path.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import ADJ, CPR, CSR, SOL, Context, DecoError, default_context


@dataclass
class SolveInfo:
    """Iterations and residuals of the last forward and adjoint solves."""
    forward: dict = field(default_factory=dict)
    adjoint: dict = field(default_factory=dict)


last = SolveInfo()


def _torch():
    import torch
    return torch


def _summary(s) -> dict:
    return dict(iter=s.iter, flag=s.flag, res_abs=s.res_abs, res_rel=s.res_rel, time_ms=s.time_ms)


def _make_function():
    torch = _torch()

    class CprSolve(torch.autograd.Function):
        @staticmethod
        def forward(fctx, values, b, r, c, prec, sol, precision, dctx):
            n = b.numel()
            A = CSR(n, n, r, c, values.detach().contiguous(), ctx=dctx)
            bd = b.detach().clone().contiguous()
            P = CPR(prec, A, bd, precision)
            S = SOL(sol, A, P, bd, precision=precision)
            last.forward = _summary(S)
            x = S.x
            fctx.save_for_backward(values, x)
            fctx.meta = (r, c, prec, sol, precision, dctx)
            return x

        @staticmethod
        def backward(fctx, gx):
            values, x = fctx.saved_tensors
            r, c, prec, sol, precision, dctx = fctx.meta
            n = x.numel()
            A = CSR(n, n, r, c, values.detach().contiguous(), ctx=dctx)
            J = ADJ(prec, A, precision)
            lam = J.solve(sol, gx.detach().to(torch.float64).contiguous())
            last.adjoint = dict(iter=J.iter, flag=J.flag, res_abs=J.res_abs, res_rel=J.res_rel, time_ms=J.time_ms)
            gA = A.grad_pattern(lam, x, -1.0) if fctx.needs_input_grad[0] else None
            gb = lam if fctx.needs_input_grad[1] else None
            return gA, gb, None, None, None, None, None, None

    return CprSolve


_fn = None


def cpr_solve(values, b, r, c, prec: dict, sol: dict, precision: int = 64, ctx: Context | None = None):
    """x = A^{-1} b with A = CSR(r, c, values) (CUDA tensors: values float64 [nnz],
    b float64 [n], r/c int32); differentiable in values and b."""
    global _fn
    torch = _torch()
    for name, t, dt in (("values", values, torch.float64), ("b", b, torch.float64), ("r", r, torch.int32),
                        ("c", c, torch.int32)):
        if not (hasattr(t, "is_cuda") and t.is_cuda and t.dtype == dt):
            raise DecoError(-1, f"{name} must be a CUDA {dt} tensor")
    if _fn is None:
        _fn = _make_function()
    return _fn.apply(values, b, r.contiguous(), c.contiguous(), prec, sol, int(precision), ctx or default_context())
