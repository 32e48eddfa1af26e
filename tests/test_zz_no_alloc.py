"""The allocation-free variable-length entry point (tridDmtsvVarlenBatchNoAlloc).

It exists for callers that cannot allocate device memory (under another
component's allocator or memory budget, or in loops that cannot absorb the
synchronisation of cudaMalloc/cudaFree); its scratch is a fixed array
compiled into the library.  Checked through the C ABI against the allocating
entry point tridDmtsvVarlenBatch on the same inputs, for two calls in a row
(the second call must not be disturbed by what the first left in the shared
array), for the size limit, and for the error word inside the array:
offsets that stop increasing make it skip systems, which
tridGetDeviceErrors must report (and then clear).  This file is named to be
collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200.varlen  # noqa: E402,F401  (registers the signatures)
from tridsolver_b200 import lib  # noqa: E402

from helpers import overlapping_varlen_problem  # noqa: E402

TOL = 1e-12  # FP64 relative max-norm, as for every FP64 solve


def _problem(seed, nsys):
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(2048), nsys))).astype(np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    total = int(off[-1])
    a = rng.uniform(-1, 1, total)
    c = rng.uniform(-1, 1, total)
    b = np.abs(a) + np.abs(c) + rng.uniform(1, 2, total)
    d = rng.standard_normal(total)
    return [torch.from_numpy(x).cuda() for x in (a, b, c, d)], torch.from_numpy(off).cuda(), total


def _call(name, a, b, c, d, off, nsys, total):
    L = lib()
    L.tridSetStream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    return getattr(L, name)(p(a), p(b), p(c), p(d), p(off), nsys, total)


def test_no_alloc_matches_allocating_entry_twice_in_a_row():
    for seed, nsys in ((11, 700), (12, 350)):
        (a, b, c, d), off, total = _problem(seed, nsys)
        d_ref, d_new = d.clone(), d.clone()
        assert _call("tridDmtsvVarlenBatch", a, b, c, d_ref, off, nsys, total) == 0
        assert _call("tridDmtsvVarlenBatchNoAlloc", a, b, c, d_new, off, nsys, total) == 0
        torch.cuda.synchronize()
        err = float((d_new - d_ref).abs().max() / d_ref.abs().max())
        assert err <= TOL, (seed, err)


def test_no_alloc_rejects_problems_beyond_its_fixed_scratch():
    a = torch.zeros(8, dtype=torch.float64, device="cuda")
    off = torch.zeros(2, dtype=torch.int64, device="cuda")
    # 10 M systems need far more than the 32 MiB the array holds
    st = _call("tridDmtsvVarlenBatchNoAlloc", a, a, a, a, off, 10_000_000, 8)
    assert st == 3  # TRID_STATUS_INVALID_VALUE


def test_no_alloc_reports_skipped_systems():
    L = lib()
    flags = ctypes.c_uint()
    assert L.tridGetDeviceErrors(ctypes.byref(flags)) == 0  # clear both words
    (a, b, c, d), off, G = overlapping_varlen_problem(22, ngood=300, npairs=200)
    a, b, c, d = [torch.from_numpy(x).cuda() for x in (a, b, c, d)]
    off_t = torch.from_numpy(off).cuda()
    nsys, total = off.size - 1, d.numel()
    d_ref, d_new = d.clone(), d.clone()
    assert _call("tridDmtsvVarlenBatch", a, b, c, d_ref, off_t, nsys, total) == 0
    assert L.tridGetDeviceErrors(ctypes.byref(flags)) == 0 and flags.value & 4
    assert _call("tridDmtsvVarlenBatchNoAlloc", a, b, c, d_new, off_t, nsys, total) == 0
    assert L.tridGetDeviceErrors(ctypes.byref(flags)) == 0
    assert flags.value & 4, flags.value  # recorded in the static array's word
    assert L.tridGetDeviceErrors(ctypes.byref(flags)) == 0 and flags.value == 0  # cleared
    # the ordinary systems (rows [0, G)) match the allocating entry point
    err = float((d_new[:G] - d_ref[:G]).abs().max() / d_ref[:G].abs().max())
    assert err <= TOL, err
