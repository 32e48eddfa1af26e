"""Parity of the scalar strided-batch solves (GPU, through the C ABI).

Mirrors the reference's file-driven GPU tests (scalar/test/test_cuda.cu:84-137:
solveX/Y/Z on the golden fixtures, FP64/FP32, opts={0,0,0}) and extends them
to the cases the reference leaves untested (Inc, padding, per-array pads,
ndim up to 8, lengths around every chunk boundary, forced methods), each
compared with the CPU oracle on the same inputs: FP64 within 1e-12 and FP32
within 1e-5 relative max-norm.
"""

import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402
from tridsolver_b200 import _lib  # noqa: E402

from helpers import RTOL, dev, host, rand_coeffs, rel_err  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
ABS_TOL = {np.float64: 1e-11, np.float32: 1e-6}   # scalar/test/utils.hpp:14-17
REL_TOL = {np.float64: 1e-11, np.float32: 1e-5}


@pytest.fixture(autouse=True)
def _auto_method():
    tb.set_method(0)
    yield
    tb.set_method(0)


def require_allclose(expected, actual, dtype):
    e = np.asarray(expected, dtype=np.float64)
    a = np.asarray(actual, dtype=np.float64)
    tol = ABS_TOL[dtype] + REL_TOL[dtype] * np.minimum(np.abs(e), np.abs(a))
    bad = np.abs(e - a) > tol
    assert not bad.any(), f"{bad.sum()} mismatches, max diff {np.abs(e - a).max()}"


def call(dtype, inc, *args):
    name = ("tridD" if dtype == np.float64 else "tridS") + "mtsvStridedBatch" + ("Inc" if inc else "")
    return getattr(tb, name)(*args)


# ---------------------------------------------------------------- golden --
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_golden_fixtures(path, dtype):
    if dtype == np.float32 and "reduced" in path:
        pytest.skip("FP64-only fixture in the reference (test_cuda_mpi.cu:289-291)")
    z = np.load(path)
    dims = [int(v) for v in z["dims"]]
    a, b, c, d = (dev(z[k].astype(dtype)) for k in "abcd")
    st = call(dtype, False, a, b, c, d, None, len(dims), int(z["solvedim"]), dims, dims)
    assert st == 0
    require_allclose(z["u"] if dtype == np.float64 else z["u_float"], host(d), dtype)


@pytest.mark.parametrize("path", [p for p in GOLDEN if "three_dim" in p or "two_dim_large" in p],
                         ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_golden_fixtures_compat_abi(path, dtype):
    """The 11-argument GPU form, called as scalar/test/test_cuda.cu:40-56 does."""
    z = np.load(path)
    dims = [int(v) for v in z["dims"]]
    a, b, c, d = (dev(z[k].astype(dtype)) for k in "abcd")
    L = tb.compat_lib()
    fn = L.tridDmtsvStridedBatch if dtype == np.float64 else L.tridSmtsvStridedBatch
    p = lambda t: t.data_ptr()
    st = fn(p(a), p(b), p(c), p(d), None, len(dims), int(z["solvedim"]), _lib.int_array(dims),
            _lib.int_array(dims), _lib.int_array([0, 0, 0]), 1)
    assert st == 0
    require_allclose(z["u"] if dtype == np.float64 else z["u_float"], host(d), dtype)


# ------------------------------------------------------- oracle parity --
def run_case(rng, dtype, dims, solvedim, pads=None, inc=False, method=None):
    pads = list(dims) if pads is None else pads
    size = int(np.prod(pads))
    a, b, c, d = rand_coeffs(rng, size, dtype)
    u = rng.standard_normal(size).astype(dtype)
    expect = oracle.mtsv(a, b, c, d, u, dims=dims, pads=pads, solvedim=solvedim, inc=inc)
    if method is not None:
        tb.set_method(*method)
    ta, tb_, tc, td, tu = (dev(x) for x in (a, b, c, d, u))
    st = call(dtype, inc, ta, tb_, tc, td, tu, len(dims), solvedim, dims, pads)
    assert st == 0
    out_d, out_u = host(td), host(tu)
    if inc:
        assert np.array_equal(out_d, d), "Inc must leave d unmodified"
        got = out_u
    else:
        assert np.array_equal(out_u, u), "non-Inc must not touch u"
        got = out_d
    # only the dims-region changes; padding is untouched
    mask = np.zeros(pads[::-1], dtype=bool)
    mask[tuple(slice(0, n) for n in dims[::-1])] = True
    base = u if inc else d
    assert np.array_equal(got.reshape(pads[::-1])[~mask], base.reshape(pads[::-1])[~mask])
    err = rel_err(got.reshape(pads[::-1])[mask], expect.reshape(pads[::-1])[mask])
    assert err <= RTOL[dtype], err
    return err


LENGTHS = [1, 2, 3, 5, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257, 511, 512,
           513, 1000]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", LENGTHS)
def test_x_lengths(dtype, n):
    run_case(np.random.default_rng(n), dtype, [n, 37], 0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", LENGTHS)
def test_y_lengths(dtype, n):
    run_case(np.random.default_rng(1000 + n), dtype, [45, n], 1)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
def test_3d_padded_inc(dtype, solvedim, inc):
    rng = np.random.default_rng(7 * solvedim + inc)
    run_case(rng, dtype, [40, 33, 27], solvedim, pads=[43, 35, 28], inc=inc)


@pytest.mark.parametrize("solvedim", [0, 1, 2, 3])
def test_4d(solvedim):
    run_case(np.random.default_rng(40 + solvedim), np.float64, [12, 9, 10, 11], solvedim,
             pads=[13, 9, 12, 11])


@pytest.mark.parametrize("solvedim", [0, 4, 7])
def test_8d(solvedim):
    run_case(np.random.default_rng(80 + solvedim), np.float64, [3, 2, 4, 2, 3, 2, 2, 5], solvedim,
             pads=[4, 2, 5, 2, 3, 3, 2, 5])


@pytest.mark.parametrize("method", [(1, 0, 0), (2, 2, 4), (2, 4, 8), (2, 8, 16), (2, 16, 4),
                                    (2, 16, 8), (2, 8, 32), (3, 8, 8), (3, 8, 32), (6, 16, 0)])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_forced_methods(method, solvedim):
    run_case(np.random.default_rng(3), np.float64, [30, 29, 28], solvedim, method=method)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [16, 48, 64, 200, 256, 512])
@pytest.mark.parametrize("inc", [False, True])
def test_x_tma_staged(dtype, n, inc):
    """Axis 0 with pads[0] a multiple of the 128-byte row: TMA-staged loads,
    and a TMA store when n fills whole rows."""
    pads0 = ((n + 31) // 32) * 32
    run_case(np.random.default_rng(n + inc), dtype, [n, 21, 3], 0, pads=[pads0, 21, 3], inc=inc)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [2, 5, 33, 64, 100, 128, 255, 256, 300, 512])
@pytest.mark.parametrize("solvedim", [1, 2])
def test_strided_tma_staged(dtype, n, solvedim):
    """Strided axes with pads[0]*sizeof a multiple of 16: TMA-staged tiles."""
    dims = [40, n, 3] if solvedim == 1 else [40, 3, n]
    run_case(np.random.default_rng(n + 7 * solvedim), dtype, dims, solvedim)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [2, 5, 16, 17, 32, 33, 64, 65, 100, 128])
@pytest.mark.parametrize("solvedim,inc", [(1, False), (2, False), (2, True)])
def test_strided_short_wide_tiles(dtype, n, solvedim, inc):
    """Short strided systems with an axis 0 of at least 64: tiles of 64
    systems x 8 chunks (FP64 up to 64 rows, FP32 up to 128) or 32 x 16; axis 0
    of 70 leaves a partial last tile."""
    dims = [70, n, 3] if solvedim == 1 else [70, 3, n]
    run_case(np.random.default_rng(n + 3 * solvedim + inc), dtype, dims, solvedim, inc=inc)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("spc", [4, 8, 16, 32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,solvedim,pads", [
    ([36, 70, 6], 1, [36, 72, 6]),
    ([36, 6, 70], 2, [40, 6, 70]),
    ([20, 3, 50, 4], 2, [24, 3, 50, 4]),
    ([16, 2, 3, 41, 2], 3, None),
    ([72, 150, 33], 2, [80, 150, 33]),    # many more tiles than CTAs, partial last x tile
    ([96, 40, 256], 2, None),             # n = 256: full 128-byte tiles, several per CTA
    ([64, 129, 7, 3], 1, None),           # rank 4, odd n
])
def test_strided_tma_spc_inc_padded(dtype, spc, inc, dims, solvedim, pads):
    """Every systems-per-CTA width of the TMA-staged strided kernels; full-line
    widths (16 FP64 / 32 FP32 systems) run the persistent streamed form, which
    loops over several tiles per CTA in the larger cases."""
    run_case(np.random.default_rng(spc + inc), dtype, dims, solvedim, pads=pads, inc=inc,
             method=(2, 0, spc))


def test_no_device_errors_recorded():
    import ctypes
    flags = ctypes.c_uint(123)
    assert tb.lib().tridGetDeviceErrors(ctypes.byref(flags)) == 0
    assert flags.value == 0


def test_padded_per_array_pads():
    rng = np.random.default_rng(11)
    dims = [20, 18, 9]
    pads = {k: [20 + i, 19 + i, 9 + i] for i, k in enumerate("abcdu")}
    host_arrs = {}
    for k in "abcdu":
        n = int(np.prod(pads[k]))
        x = rng.uniform(-1, 1, n)
        if k == "b":
            x = 3.0 + rng.uniform(0, 1, n)
        host_arrs[k] = x
    for solvedim in range(3):
        for inc in (False, True):
            ap = tuple(pads[k] for k in "abcdu")
            expect = oracle.mtsv(*(host_arrs[k] for k in "abcd"), host_arrs["u"], dims=dims,
                                 solvedim=solvedim, inc=inc, array_pads=ap)
            t = {k: dev(host_arrs[k]) for k in "abcdu"}
            fn = tb.tridDmtsvStridedBatchPaddedInc if inc else tb.tridDmtsvStridedBatchPadded
            st = fn(t["a"], pads["a"], t["b"], pads["b"], t["c"], pads["c"], t["d"], pads["d"],
                    t["u"], pads["u"], 3, solvedim, dims, opts=[0, 0, 0], sync=1)
            assert st == 0
            got = t["u"] if inc else t["d"]
            assert rel_err(host(got), expect) <= 1e-12


@pytest.mark.parametrize("solvedim", [0, 1])
def test_a0_and_cn_never_read(solvedim):
    rng = np.random.default_rng(5)
    dims = [70, 50]
    a, b, c, d = rand_coeffs(rng, 3500)
    A, C = a.reshape(50, 70).copy(), c.reshape(50, 70).copy()
    if solvedim == 0:
        A[:, 0], C[:, -1] = np.nan, np.inf
    else:
        A[0, :], C[-1, :] = np.nan, np.inf
    expect = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
    td = dev(d)
    assert tb.tridDmtsvStridedBatch(dev(A.ravel()), dev(b), dev(C.ravel()), td, None, 2, solvedim,
                                    dims, dims) == 0
    got = host(td)
    assert np.isfinite(got).all()
    assert rel_err(got, expect) <= 1e-12


def test_empty_problem_is_a_noop():
    d = torch.ones(10, dtype=torch.float64, device="cuda")
    assert tb.tridDmtsvStridedBatch(d, d, d, d, None, 2, 0, [0, 10], [0, 10]) == 0
    assert tb.tridDmtsvStridedBatch(d, d, d, d, None, 2, 1, [10, 0], [10, 0]) == 0
    assert torch.all(d == 1)


def test_solve_on_side_stream():
    rng = np.random.default_rng(2)
    a, b, c, d = rand_coeffs(rng, 64 * 300)
    expect = oracle.mtsv(a, b, c, d, dims=[300, 64], solvedim=0)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ta, tb_, tc, td = (dev(x) for x in (a, b, c, d))
        tb.solve(ta.view(64, 300), tb_.view(64, 300), tc.view(64, 300), td.view(64, 300), dim=-1)
    s.synchronize()
    assert rel_err(td.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_full_cube_256_fp64(solvedim):
    """The benchmark workload (256^3, FP64) against the oracle."""
    run_case(np.random.default_rng(256 + solvedim), np.float64, [256, 256, 256], solvedim)


def test_full_cube_256_fp32_residual():
    rng = np.random.default_rng(9)
    for solvedim in range(3):
        run_case(rng, np.float32, [256, 256, 256], solvedim)
