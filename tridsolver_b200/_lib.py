"""ctypes bindings of the tridsolver_b200 C ABI (include/*.h).

The shared libraries are built in-tree by ``python -m tridsolver_b200.build``.
There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_MAIN = os.path.join(HERE, "libtridb200.so")
LIB_COMPAT = os.path.join(HERE, "libtridb200_cudacompat.so")

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_flt = ctypes.c_float
vp = ctypes.c_void_p
ip = ctypes.POINTER(ctypes.c_int)

STATUS_NAMES = {
    0: "TRID_STATUS_SUCCESS",
    1: "TRID_STATUS_NOT_INITIALIZED",
    2: "TRID_STATUS_ALLOC_FAILED",
    3: "TRID_STATUS_INVALID_VALUE",
    4: "TRID_STATUS_ARCH_MISMATCH",
    5: "TRID_STATUS_MAPPING_ERROR",
    6: "TRID_STATUS_EXECUTION_FAILED",
    7: "TRID_STATUS_INTERNAL_ERROR",
    8: "TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED",
    9: "TRID_STATUS_ZERO_PIVOT",
}

_SCALAR9 = [vp, vp, vp, vp, vp, c_int, c_int, ip, ip]
_SCALAR11 = _SCALAR9 + [ip, c_int]
_PADDED = [vp, ip, vp, ip, vp, ip, vp, ip, vp, ip, c_int, c_int, ip, ip, c_int]

# name -> (restype, argtypes) for the symbols every library exports
_ADJ = [vp, vp, vp, vp, vp, vp, vp, vp, vp, c_int, c_int, ip, ip]
_FWDADJ = [vp] * 10 + [c_int, c_int, ip, ip]
_SPLIT_REDUCE = [vp, vp, vp, vp, c_int, c_int, ip, ip, vp]
_SPLIT_FINISH = [vp, vp, vp, vp, vp, c_int, c_int, ip, ip, vp, c_int, c_int, c_int]

_COMMON = {
    "tridDmtsvStridedBatchAdjoint": (c_int, _ADJ),
    "tridSmtsvStridedBatchAdjoint": (c_int, _ADJ),
    "tridDmtsvStridedBatchFwdAdj": (c_int, _FWDADJ),
    "tridDmtsvStridedBatchOut": (c_int, [vp] * 5 + [c_int, c_int, ip, ip]),
    "tridSmtsvStridedBatchOut": (c_int, [vp] * 5 + [c_int, c_int, ip, ip]),
    "tridSmtsvStridedBatchFwdAdj": (c_int, _FWDADJ),
    "tridDmtsvStridedBatchSplitReduce": (c_int, _SPLIT_REDUCE),
    "tridSmtsvStridedBatchSplitReduce": (c_int, _SPLIT_REDUCE),
    "tridDmtsvStridedBatchSplitFinish": (c_int, _SPLIT_FINISH),
    "tridSmtsvStridedBatchSplitFinish": (c_int, _SPLIT_FINISH),
    "tridDmtsvStridedBatchPadded": (c_int, _PADDED),
    "tridDmtsvStridedBatchPaddedInc": (c_int, _PADDED),
    "tridSmtsvStridedBatchPadded": (c_int, _PADDED),
    "tridSmtsvStridedBatchPaddedInc": (c_int, _PADDED),
    "initTridMultiDimBatchSolve": (None, [c_int, ip, ip]),
    "tridSetStream": (c_int, [vp]),
    "tridGetStream": (vp, []),
    "tridReleaseScratch": (c_int, []),
    "tridGetStatusString": (ctypes.c_char_p, [c_int]),
    "tridSetMethod": (c_int, [c_int, c_int, c_int]),
    "tridGetDeviceErrors": (c_int, [ctypes.POINTER(ctypes.c_uint)]),
    "tridLoadTuningTable": (c_int, [ctypes.c_char_p]),
    "tridQueryMethod": (c_int, [c_int, c_int, c_int, ip, ip, ip]),
}
_MAIN_ONLY = {
    "tridSmtsvStridedBatch": (c_int, _SCALAR9),
    "tridDmtsvStridedBatch": (c_int, _SCALAR9),
    "tridSmtsvStridedBatchInc": (c_int, _SCALAR9),
    "tridDmtsvStridedBatchInc": (c_int, _SCALAR9),
    "tridCmtsvStridedBatch": (c_int, _SCALAR9),
    "tridCmtsvStridedBatchInc": (c_int, _SCALAR9),
    "tridZmtsvStridedBatch": (c_int, _SCALAR9),
    "tridZmtsvStridedBatchInc": (c_int, _SCALAR9),
    "tridSmtsvStridedBatchMixed": (c_int, _SCALAR9),
    "tridSmtsvStridedBatchMixedInc": (c_int, _SCALAR9),
}
_COMPAT_ONLY = {
    "tridSmtsvStridedBatch": (c_int, _SCALAR11),
    "tridDmtsvStridedBatch": (c_int, _SCALAR11),
    "tridSmtsvStridedBatchInc": (c_int, _SCALAR11),
    "tridDmtsvStridedBatchInc": (c_int, _SCALAR11),
}

_cache = {}


class TridError(RuntimeError):
    """A tridsolver_b200 call returned a status other than SUCCESS."""

    def __init__(self, status, what=""):
        self.status = int(status)
        super().__init__(f"{what}: {STATUS_NAMES.get(self.status, self.status)}")


def _load(path, table):
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise RuntimeError(f"{os.path.basename(path)} is not built; run "
                           "`python -m tridsolver_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in table.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _cache[path] = lib
    return lib


def register(table_main, table_both=None):
    """Add signatures of further entry points (used by the component modules)."""
    _MAIN_EXTRA.update(table_main)
    if table_both:
        _COMMON.update(table_both)


_MAIN_EXTRA = {}


def lib():
    """libtridb200.so (9-argument strided batch + every extension)."""
    return _load(LIB_MAIN, {**_COMMON, **_MAIN_ONLY, **_MAIN_EXTRA})


def compat_lib():
    """libtridb200_cudacompat.so (11-argument strided batch)."""
    return _load(LIB_COMPAT, {**_COMMON, **_COMPAT_ONLY})


def int_array(vals):
    vals = [int(v) for v in vals]
    return (c_int * max(1, len(vals)))(*vals)
