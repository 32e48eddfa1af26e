"""torch.autograd.Function over the C ABI: a differentiable batched solve.

``trid_solve(a, b, c, d, dim=-1)`` returns x with A x = d along torch
dimension ``dim`` (A tridiagonal with sub-diagonal a, diagonal b,
super-diagonal c; a[0] and c[n-1] of every system unused).  The forward pass
is the out-of-place solve tridDmtsvStridedBatchOut / tridSmtsvStridedBatchOut
(x written next to d, which autograd keeps, so no copy of d); the backward
pass is one call of the hand-written adjoint kernel
(tridXmtsvStridedBatchAdjoint): it solves A^T g = dL/dx in place and forms
dL/da_i = -g_i x_{i-1}, dL/db_i = -g_i x_i, dL/dc_i = -g_i x_{i+1},
dL/dd = g in the same pass.
"""

import torch

from ._lib import TridError
from .scalar import (tridDmtsvStridedBatchAdjoint, tridDmtsvStridedBatchOut,
                     tridSmtsvStridedBatchAdjoint, tridSmtsvStridedBatchOut)


def _layout(t, dim):
    ndim = t.dim()
    dim = dim % ndim
    dims = list(reversed(t.shape))
    return ndim, ndim - 1 - dim, dims


class TridSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, b, c, d, dim):
        a, b, c, d = (t.contiguous() for t in (a, b, c, d))
        if not (a.shape == b.shape == c.shape == d.shape):
            raise ValueError("a, b, c, d must have one shape")
        if d.dtype not in (torch.float32, torch.float64) or not d.is_cuda:
            raise TypeError("CUDA float32/float64 tensors only")
        x = torch.empty_like(d)
        ndim, sd, dims = _layout(x, dim)
        fn = tridDmtsvStridedBatchOut if x.dtype == torch.float64 else tridSmtsvStridedBatchOut
        st = fn(a, b, c, d, x, ndim, sd, dims, dims)
        if st != 0:
            raise TridError(st, fn.__name__)
        ctx.save_for_backward(a, b, c, x)
        ctx.dim = dim
        return x

    @staticmethod
    def backward(ctx, w):
        a, b, c, x = ctx.saved_tensors
        w = w.contiguous()
        ndim, sd, dims = _layout(x, ctx.dim)
        need = ctx.needs_input_grad
        outs = [torch.empty_like(x) if need[i] else None for i in range(4)]
        fn = (tridDmtsvStridedBatchAdjoint if x.dtype == torch.float64
              else tridSmtsvStridedBatchAdjoint)
        st = fn(a, b, c, x, w, outs[0], outs[1], outs[2], outs[3], ndim, sd, dims, dims)
        if st != 0:
            raise TridError(st, fn.__name__)
        return outs[0], outs[1], outs[2], outs[3], None


def trid_solve(a, b, c, d, dim=-1):
    """Differentiable batched tridiagonal solve along torch dimension ``dim``."""
    return TridSolve.apply(a, b, c, d, dim)
