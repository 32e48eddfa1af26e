"""Variable-length packed batches over the C ABI (tridXmtsvVarlenBatch).

``solve_varlen(a, b, c, d, offsets)``: system s occupies
``[offsets[s], offsets[s+1])`` of the 1-D CUDA tensors a, b, c, d (int64
offsets on the GPU); the solution overwrites d.  Up to 8192 rows per system.
"""

import ctypes

import torch

from ._lib import TridError, c_int, lib, register, vp
from .scalar import _bind_stream, _ptr, _real_dtype

c_ll = ctypes.c_longlong
register({
    "tridDmtsvVarlenBatch": (c_int, [vp, vp, vp, vp, vp, c_ll, c_ll]),
    "tridSmtsvVarlenBatch": (c_int, [vp, vp, vp, vp, vp, c_ll, c_ll]),
    "tridDmtsvVarlenBatchNoAlloc": (c_int, [vp, vp, vp, vp, vp, c_ll, c_ll]),
})


def solve_varlen(a, b, c, d, offsets, total=None):
    dt = _real_dtype(a, b, c, d)
    if offsets.dtype != torch.int64 or not offsets.is_cuda:
        raise TypeError("offsets: int64 CUDA tensor of nsys+1 entries")
    nsys = offsets.numel() - 1
    total = d.numel() if total is None else int(total)
    L = lib()
    _bind_stream(L)
    fn = L.tridDmtsvVarlenBatch if dt == torch.float64 else L.tridSmtsvVarlenBatch
    st = fn(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(offsets), nsys, total)
    if st != 0:
        raise TridError(st, fn.__name__)
    return d
