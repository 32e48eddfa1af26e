"""tridsolver_b200 -- B200-native batched tridiagonal solvers.

The product is the C ABI in ``include/*.h`` (libtridb200.so and
libtridb200_cudacompat.so, hand-written sm_100a CUDA).  This package is the
Python host side over that ABI:

* the reference's entry points under the reference's names
  (``tridDmtsvStridedBatch`` ... with ``(a, b, c, d, u, ndim, solvedim, dims,
  pads)``, returning a tridStatus_t), taking CUDA tensors or raw device
  pointers -- scalar/include/trid_cpu.h:53-82, trid_cuda.h:44-80;
* ``solve``: the same solve on torch tensors, raising ``TridError``;
* component modules: ``block`` (block tridiagonal), ``adjoint`` (autograd),
  ``varlen`` (packed variable-length batches), ``adi`` (heat-diffusion step),
  ``autotune``.

Calls are enqueued on torch's current CUDA stream.  There is no CPU fallback:
without the built library every call raises.
"""

from . import _lib
from ._lib import STATUS_NAMES, TridError, compat_lib, lib  # noqa: F401
from .scalar import (  # noqa: F401
    initTridMultiDimBatchSolve,
    solve,
    tridCmtsvStridedBatch,
    tridCmtsvStridedBatchInc,
    tridDmtsvStridedBatch,
    tridDmtsvStridedBatchAdjoint,
    tridSmtsvStridedBatchAdjoint,
    tridDmtsvStridedBatchFwdAdj,
    tridSmtsvStridedBatchFwdAdj,
    tridDmtsvStridedBatchOut,
    tridSmtsvStridedBatchOut,
    solve_fwd_adj,
    tridDmtsvStridedBatchInc,
    tridDmtsvStridedBatchPadded,
    tridDmtsvStridedBatchPaddedInc,
    tridSmtsvStridedBatch,
    tridSmtsvStridedBatchInc,
    tridSmtsvStridedBatchPadded,
    tridSmtsvStridedBatchPaddedInc,
    tridSmtsvStridedBatchMixed,
    tridSmtsvStridedBatchMixedInc,
    tridZmtsvStridedBatch,
    tridZmtsvStridedBatchInc,
    set_method,
)
from .autograd import TridSolve, trid_solve  # noqa: F401
from . import adi, block, varlen  # noqa: F401
