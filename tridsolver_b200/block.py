"""Block-tridiagonal batched solve over the C ABI (include/blktrid_b200.h).

Arrays use the reference GPU's interleaved layout: A, B, C of shape
(N, P, M, M) and d, x of shape (N, P, M), contiguous, on the GPU.
``btsv`` is the reference's dbtsv_gpu/sbtsv_gpu with a status;
``btsv_adjoint`` returns the gradients of a loss through the solve.
"""

import ctypes

import torch

from ._lib import TridError, c_int, lib, register, vp
from .scalar import _bind_stream, _ptr, _real_dtype

_BT = [vp, vp, vp, vp, vp, c_int, c_int, c_int, vp, vp]
_BTA = [vp, vp, vp, vp, vp, vp, vp, vp, vp, c_int, c_int, c_int]
register({
    "tridDbtsvBatch": (c_int, _BT),
    "tridSbtsvBatch": (c_int, _BT),
    "tridDbtsvBatchAdjoint": (c_int, _BTA),
    "tridSbtsvBatchAdjoint": (c_int, _BTA),
})


def _shape(A, d):
    if A.dim() != 4 or A.shape[2] != A.shape[3] or d.shape != A.shape[:3]:
        raise ValueError("A/B/C must be (N, P, M, M) and d (N, P, M)")
    return int(A.shape[0]), int(A.shape[1]), int(A.shape[2])


def btsv(A, B, C, d, x=None, Cstar=None, dstar=None):
    """Solve the block systems; returns x (new tensor unless given)."""
    N, P, M = _shape(A, d)
    dt = _real_dtype(A, B, C, d, x, Cstar, dstar)
    x = torch.empty_like(d) if x is None else x
    L = lib()
    _bind_stream(L)
    fn = L.tridDbtsvBatch if dt == torch.float64 else L.tridSbtsvBatch
    st = fn(_ptr(A), _ptr(B), _ptr(C), _ptr(d), _ptr(x), N, P, M, _ptr(Cstar), _ptr(dstar))
    if st != 0:
        raise TridError(st, fn.__name__)
    return x


def btsv_adjoint(A, B, C, u, w, need=(True, True, True, True)):
    """Gradients (dA, dB, dC, dd) of a loss with dL/dx = w at the solution u."""
    N, P, M = _shape(A, u)
    dt = _real_dtype(A, B, C, u, w)
    outs = [torch.empty_like(t) if k else None for k, t in zip(need, (A, B, C, u))]
    L = lib()
    _bind_stream(L)
    fn = L.tridDbtsvBatchAdjoint if dt == torch.float64 else L.tridSbtsvBatchAdjoint
    st = fn(_ptr(A), _ptr(B), _ptr(C), _ptr(u), _ptr(w), *[_ptr(o) for o in outs], N, P, M)
    if st != 0:
        raise TridError(st, fn.__name__)
    return tuple(outs)


class BlockTridSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, B, C, d):
        A, B, C, d = (t.contiguous() for t in (A, B, C, d))
        x = btsv(A, B, C, d)
        ctx.save_for_backward(A, B, C, x)
        return x

    @staticmethod
    def backward(ctx, w):
        A, B, C, x = ctx.saved_tensors
        return btsv_adjoint(A, B, C, x, w.contiguous(), tuple(ctx.needs_input_grad[:4]))


def block_trid_solve(A, B, C, d):
    """Differentiable block-tridiagonal solve (interleaved layout)."""
    return BlockTridSolve.apply(A, B, C, d)
