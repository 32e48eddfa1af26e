"""Variable-length packed batches (GPU): one persistent launch, compared with
the oracle's per-system Thomas (oracle_varlen, pinned to the reference's
trid_scalarD).  FP64 1e-12, FP32 1e-5 relative max-norm per system."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from tridsolver_b200.varlen import solve_varlen  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import overlapping_varlen_problem, rand_coeffs  # noqa: E402


def run(lens, dtype=np.float64, seed=0):
    rng = np.random.default_rng(seed)
    lens = np.asarray(lens, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    total = int(off[-1])
    a, b, c, d = rand_coeffs(rng, total, dtype)
    expect = oracle.varlen(a, b, c, d, off)
    t = [torch.from_numpy(x).cuda() for x in (a, b, c, d)]
    solve_varlen(*t, torch.from_numpy(off).cuda())
    got = t[3].cpu().numpy()
    tol = 1e-12 if dtype == np.float64 else 1e-5
    for s in range(len(lens)):
        o, n = off[s], lens[s]
        if n == 0:
            continue
        ref = expect[o:o + n]
        err = np.abs(got[o:o + n] - ref).max() / max(np.abs(ref).max(), 1e-300)
        assert err <= tol, (s, n, err)


def test_edge_lengths():
    run([1, 2, 3, 31, 32, 33, 64, 65, 128, 129, 255, 256, 257, 511, 512, 513, 1000, 4096, 8191,
         8192, 5, 0, 7])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_log_uniform_lengths(dtype):
    rng = np.random.default_rng(42)
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(8192), 3000))).astype(np.int64)
    run(lens, dtype, seed=1)


def test_many_short_systems():
    rng = np.random.default_rng(3)
    run(rng.integers(1, 200, 20000), seed=2)


def test_rejects_and_flags():
    flags = ctypes.c_uint()
    tb.lib().tridGetDeviceErrors(ctypes.byref(flags))  # clear
    # a system longer than 8192 rows is skipped and flagged, the rest solved
    rng = np.random.default_rng(5)
    lens = np.array([100, 9000, 300], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    a, b, c, d = rand_coeffs(rng, int(off[-1]))
    expect = oracle.varlen(a, b, c, d, off)
    t = [torch.from_numpy(x).cuda() for x in (a, b, c, d)]
    solve_varlen(*t, torch.from_numpy(off).cuda())
    got = t[3].cpu().numpy()
    assert np.allclose(got[:100], expect[:100], rtol=1e-12, atol=1e-12)
    assert np.array_equal(got[100:9100], d[100:9100])
    assert np.allclose(got[9100:], expect[9100:], rtol=1e-12, atol=1e-12)
    tb.lib().tridGetDeviceErrors(ctypes.byref(flags))
    assert flags.value & 8
    # decreasing offsets: that system is skipped and flagged
    off2 = torch.tensor([0, 50, 40, 90], dtype=torch.int64, device="cuda")
    dd = torch.ones(90, dtype=torch.float64, device="cuda")
    bb = torch.full((90,), 3.0, dtype=torch.float64, device="cuda")
    solve_varlen(dd, bb, dd, dd.clone(), off2)
    torch.cuda.synchronize()
    tb.lib().tridGetDeviceErrors(ctypes.byref(flags))
    assert flags.value & 4


def test_non_monotone_offsets_past_capacity_are_skipped():
    """Offsets that stop increasing: the decreasing systems are skipped and
    flagged (bit 4), the valid-looking ones (all overlapping the same 8192
    rows) go to the long-system CTAs without any table passing nsys, nothing
    is written out of bounds, and the ordinary systems before them are
    solved."""
    flags = ctypes.c_uint()
    tb.lib().tridGetDeviceErrors(ctypes.byref(flags))  # clear
    (a, b, c, d), off, G = overlapping_varlen_problem(21)
    expect = oracle.varlen(a[:G], b[:G], c[:G], d[:G], off[:601])
    t = [torch.from_numpy(x).cuda() for x in (a, b, c, d)]
    solve_varlen(*t, torch.from_numpy(off).cuda())
    got = t[3].cpu().numpy()
    for s in range(600):
        o, n = off[s], off[s + 1] - off[s]
        ref = expect[o:o + n]
        err = np.abs(got[o:o + n] - ref).max() / max(np.abs(ref).max(), 1e-300)
        assert err <= 1e-12, (s, n, err)
    assert np.isfinite(got).all()
    tb.lib().tridGetDeviceErrors(ctypes.byref(flags))
    assert flags.value & 4
    assert not flags.value & 1  # no finish wait gave up
