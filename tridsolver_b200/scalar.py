"""Scalar strided-batch solves: the reference's API names over the C ABI.

Each ``trid?mtsvStridedBatch*`` function takes the reference's arguments
(scalar/include/trid_cpu.h:53-82; Padded forms trid_cuda.h:61-84) with CUDA
tensors (or integer device pointers) for the arrays and Python sequences for
dims/pads, and returns the tridStatus_t the C ABI returned -- the same
contract as the reference, whose callers check the status.  ``solve`` is the
torch-facing convenience that raises ``TridError`` instead.
"""

import ctypes

from ._lib import TridError, int_array, lib

try:  # torch is only needed for tensor arguments and the current stream
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    if torch is not None and isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise ValueError("tridsolver_b200 works on CUDA tensors (device pointers)")
        return ctypes.c_void_p(x.data_ptr())
    raise TypeError(f"expected a CUDA tensor or a device pointer, got {type(x)}")


def _real_dtype(*tensors):
    """The common element type of the given tensors (None entries skipped),
    float32 or float64; anything else raises TypeError before any call."""
    dts = {t.dtype for t in tensors if t is not None}
    if len(dts) != 1 or next(iter(dts)) not in (torch.float32, torch.float64):
        raise TypeError(f"float32 or float64 tensors of one dtype only, got {sorted(map(str, dts))}")
    return next(iter(dts))


def _bind_stream(L):
    if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
        L.tridSetStream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _scalar9(name):
    def f(a, b, c, d, u, ndim, solvedim, dims, pads):
        L = lib()
        _bind_stream(L)
        return getattr(L, name)(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(u), int(ndim),
                                int(solvedim), int_array(dims), int_array(pads))
    f.__name__ = name
    f.__doc__ = f"{name}(a, b, c, d, u, ndim, solvedim, dims, pads) -> tridStatus_t"
    return f


def _padded(name):
    def f(a, a_pads, b, b_pads, c, c_pads, d, d_pads, u, u_pads, ndim, solvedim, dims,
          opts=None, sync=0):
        L = lib()
        _bind_stream(L)
        return getattr(L, name)(_ptr(a), int_array(a_pads), _ptr(b), int_array(b_pads), _ptr(c),
                                int_array(c_pads), _ptr(d), int_array(d_pads), _ptr(u),
                                int_array(u_pads if u_pads is not None else d_pads), int(ndim),
                                int(solvedim), int_array(dims),
                                int_array(opts) if opts is not None else None, int(sync))
    f.__name__ = name
    return f


tridSmtsvStridedBatch = _scalar9("tridSmtsvStridedBatch")
tridDmtsvStridedBatch = _scalar9("tridDmtsvStridedBatch")
tridSmtsvStridedBatchInc = _scalar9("tridSmtsvStridedBatchInc")
tridDmtsvStridedBatchInc = _scalar9("tridDmtsvStridedBatchInc")
# complex element types (the reference's commented-out tridC/ZmtsvStridedBatch,
# trid_cuda.cu:546-600) and FP32 storage with FP64 arithmetic
tridCmtsvStridedBatch = _scalar9("tridCmtsvStridedBatch")
tridCmtsvStridedBatchInc = _scalar9("tridCmtsvStridedBatchInc")
tridZmtsvStridedBatch = _scalar9("tridZmtsvStridedBatch")
tridZmtsvStridedBatchInc = _scalar9("tridZmtsvStridedBatchInc")
tridSmtsvStridedBatchMixed = _scalar9("tridSmtsvStridedBatchMixed")
tridSmtsvStridedBatchMixedInc = _scalar9("tridSmtsvStridedBatchMixedInc")
tridSmtsvStridedBatchPadded = _padded("tridSmtsvStridedBatchPadded")
tridDmtsvStridedBatchPadded = _padded("tridDmtsvStridedBatchPadded")
tridSmtsvStridedBatchPaddedInc = _padded("tridSmtsvStridedBatchPaddedInc")
tridDmtsvStridedBatchPaddedInc = _padded("tridDmtsvStridedBatchPaddedInc")


def _adjoint(name):
    def f(a, b, c, u, w, da, db, dc, dd, ndim, solvedim, dims, pads):
        L = lib()
        _bind_stream(L)
        return getattr(L, name)(_ptr(a), _ptr(b), _ptr(c), _ptr(u), _ptr(w), _ptr(da), _ptr(db),
                                _ptr(dc), _ptr(dd), int(ndim), int(solvedim), int_array(dims),
                                int_array(pads))
    f.__name__ = name
    f.__doc__ = (f"{name}(a, b, c, u, w, da, db, dc, dd, ndim, solvedim, dims, pads) -> status: "
                 "gradients of a strided-batch solve (outputs may be None)")
    return f


tridDmtsvStridedBatchAdjoint = _adjoint("tridDmtsvStridedBatchAdjoint")
tridSmtsvStridedBatchAdjoint = _adjoint("tridSmtsvStridedBatchAdjoint")


def _fwdadj(name):
    def f(a, b, c, d, w, x, da, db, dc, dd, ndim, solvedim, dims, pads):
        L = lib()
        _bind_stream(L)
        return getattr(L, name)(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(w), _ptr(x), _ptr(da),
                                _ptr(db), _ptr(dc), _ptr(dd), int(ndim), int(solvedim),
                                int_array(dims), int_array(pads))
    f.__name__ = name
    f.__doc__ = (f"{name}(a, b, c, d, w, x, da, db, dc, dd, ndim, solvedim, dims, pads) -> "
                 "status: x = A^{-1} d and the gradients of <w, x> in one call")
    return f


def _out(name):
    def f(a, b, c, d, x, ndim, solvedim, dims, pads):
        L = lib()
        _bind_stream(L)
        return getattr(L, name)(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(x), int(ndim),
                                int(solvedim), int_array(dims), int_array(pads))
    f.__name__ = name
    f.__doc__ = (f"{name}(a, b, c, d, x, ndim, solvedim, dims, pads) -> status: "
                 "x = A^{-1} d, d left intact")
    return f


tridDmtsvStridedBatchOut = _out("tridDmtsvStridedBatchOut")
tridSmtsvStridedBatchOut = _out("tridSmtsvStridedBatchOut")

tridDmtsvStridedBatchFwdAdj = _fwdadj("tridDmtsvStridedBatchFwdAdj")
tridSmtsvStridedBatchFwdAdj = _fwdadj("tridSmtsvStridedBatchFwdAdj")


def solve_fwd_adj(a, b, c, d, w, dim=-1):
    """x = A^{-1} d along torch dimension ``dim`` and the gradients of the
    linear loss sum(w * x) with respect to a, b, c, d, from one call (one
    kernel for the unit-stride axis up to 4096 rows).  Returns
    (x, (da, db, dc, dd)); the inputs are left unchanged."""
    shape = tuple(d.shape)
    for t in (a, b, c, d, w):
        if tuple(t.shape) != shape or t.dtype != d.dtype or not t.is_contiguous():
            raise ValueError("a, b, c, d, w must be contiguous tensors of one shape/dtype")
    ndim = len(shape)
    dim = dim % ndim
    dims = list(reversed(shape))
    if d.dtype == torch.float64:
        fn = tridDmtsvStridedBatchFwdAdj
    elif d.dtype == torch.float32:
        fn = tridSmtsvStridedBatchFwdAdj
    else:
        raise TypeError("float32 or float64 only")
    x = torch.empty_like(d)
    grads = [torch.empty_like(d) for _ in range(4)]
    st = fn(a, b, c, d, w, x, *grads, ndim, ndim - 1 - dim, dims, dims)
    if st != 0:
        raise TridError(st, fn.__name__)
    return x, tuple(grads)


def initTridMultiDimBatchSolve(ndim, dims, pads):
    lib().initTridMultiDimBatchSolve(int(ndim), int_array(dims), int_array(pads))


def set_method(method=0, chunk=0, sys_per_cta=0):
    """Force the algorithm for calls from this thread (0 = automatic)."""
    st = lib().tridSetMethod(int(method), int(chunk), int(sys_per_cta))
    if st != 0:
        raise TridError(st, "tridSetMethod")


def solve(a, b, c, d, dim=-1, u=None, inc=False, fp64_arithmetic=False):
    """Solve the tridiagonal systems along torch dimension ``dim``.

    a, b, c, d (and u for ``inc``) are contiguous CUDA tensors of one shape
    and dtype (float32, float64, complex64 or complex128).
    ``fp64_arithmetic`` (float32 only) solves in FP64 and rounds each result
    to float32 once.  Without ``inc`` the solution overwrites
    ``d`` (returned); with ``inc`` it is added to ``u`` (returned) and ``d``
    is left unchanged.  Torch's dimension k is the library's axis ndim-1-k
    (the last torch dimension is the unit-stride axis 0).
    """
    shape = tuple(d.shape)
    for t in (a, b, c, d) + ((u,) if inc else ()):
        if tuple(t.shape) != shape or t.dtype != d.dtype or not t.is_contiguous():
            raise ValueError("a, b, c, d (and u) must be contiguous tensors of one shape/dtype")
    if inc and u is None:
        raise ValueError("inc=True needs u")
    ndim = len(shape)
    if ndim == 0:
        raise ValueError("need at least one dimension")
    dim = dim % ndim
    dims = list(reversed(shape))
    solvedim = ndim - 1 - dim
    fns = {
        torch.float64: (tridDmtsvStridedBatch, tridDmtsvStridedBatchInc),
        torch.float32: ((tridSmtsvStridedBatchMixed, tridSmtsvStridedBatchMixedInc)
                        if fp64_arithmetic else (tridSmtsvStridedBatch, tridSmtsvStridedBatchInc)),
        torch.complex128: (tridZmtsvStridedBatch, tridZmtsvStridedBatchInc),
        torch.complex64: (tridCmtsvStridedBatch, tridCmtsvStridedBatchInc),
    }
    if d.dtype not in fns:
        raise TypeError("float32, float64, complex64 or complex128 only")
    if fp64_arithmetic and d.dtype != torch.float32:
        raise TypeError("fp64_arithmetic applies to float32 tensors")
    fn = fns[d.dtype][1 if inc else 0]
    st = fn(a, b, c, d, u, ndim, solvedim, dims, dims)
    if st != 0:
        raise TridError(st, fn.__name__)
    return u if inc else d
