"""torch.autograd binding of the solve x = A^{-1} b over the C ABI.

Forward: SPAI build of M on A's pattern + BiCGSTAB (dcu_spai_solve_d).
Backward (hand-written adjoint): A^T lambda = dL/dx solved by BiCGSTAB with
preconditioner M^T (dcu_bicgstab_transpose_d); then dL/db = lambda and
dL/dA_ij = -lambda_i x_j on A's pattern (dcu_sampled_outer_d).  M changes the
iteration, not the solution, so the gradient needs no derivative of M.
"""
from __future__ import annotations

import torch

from .api import Context


class SpaiSolve(torch.autograd.Function):
    @staticmethod
    def forward(fctx, val, b, ptr, idx, ctx: Context, opts: dict):
        n, nnz = b.numel(), val.numel()
        x = torch.zeros_like(b)
        mval = torch.zeros_like(val)
        bi, si = ctx.solve_d(n, nnz, ptr, idx, val.detach().contiguous(), b.detach().contiguous(), x, mval_d=mval,
                             **opts)
        if si.status != 0:
            raise RuntimeError(f"forward solve did not converge (status {si.status}, {si.iters} iterations)")
        fctx.save_for_backward(val, x, mval, ptr, idx)
        fctx.dcu = (ctx, opts)
        return x

    @staticmethod
    def backward(fctx, gx):
        val, x, mval, ptr, idx = fctx.saved_tensors
        ctx, opts = fctx.dcu
        n, nnz = x.numel(), val.numel()
        lam = torch.zeros_like(x)
        si = ctx.bicgstab_transpose_d(n, nnz, ptr, idx, val.detach().contiguous(), mval, gx.contiguous(), lam,
                                      **opts)
        if si.status != 0:
            raise RuntimeError(f"adjoint solve did not converge (status {si.status}, {si.iters} iterations)")
        dval = torch.empty_like(val)
        ctx.sampled_outer_d(n, nnz, ptr, idx, lam, x, -1.0, dval)
        return dval, lam, None, None, None, None


def spai_solve(val, b, ptr, idx, ctx: Context, **opts):
    """x = A^{-1} b for the CSC matrix (ptr, idx, val), differentiable in val and b."""
    return SpaiSolve.apply(val, b, ptr, idx, ctx, opts)
