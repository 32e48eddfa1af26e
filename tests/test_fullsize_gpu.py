"""Parity at the benchmark sizes (GPU, through the C ABI).

The other GPU tests compare with the plain-C restatement of the reference
(oracle/trid_oracle.c) at sizes the restatement finishes quickly.  These run
the workloads at their full benchmark sizes and compare against the
reference's own CPU code where it exists:

* the 256^3 cube along each axis, FP64 and FP32, against the reference's
  tridD/SmtsvStridedBatch (scalar/src/cpu/trid_cpu.cpp:535-595, compiled
  unmodified into oracle/_ref) on the same inputs, and on sampled systems
  against FP64 dense LU;
* the padded single-precision forms tridSmtsvStridedBatchPadded[Inc];
* the block batch N = 256, P = 32,768, M = 2, 4, 8, forward and adjoint:
  the whole batch solved on the GPU, 256 sampled systems checked against the
  corrected block-Thomas oracle (the reference's blktrid_cpu.cpp:388-495
  with its matrix product fixed);
* the variable-length batch of 200,000 systems with lengths log-uniform on
  [8, 8192], sampled systems checked against the reference's trid_scalarD
  (trid_cpu.cpp:597-602) one system at a time.

Bars: FP64 1e-12, FP32 1e-5 relative max-norm (and 1e-5 for FP32 against the
FP64 dense LU).  Inputs of the batched workloads are drawn on the GPU from a
seeded generator and copied back for the checks.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from tridsolver_b200 import block  # noqa: E402
from tridsolver_b200.varlen import solve_varlen  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import RTOL, dev, host, rand_coeffs, rel_err  # noqa: E402

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference CPU library (oracle/_ref) not built")


@pytest.fixture(autouse=True)
def _free_memory():
    tb.set_method(0)
    yield
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def cube_inputs(seed, dtype, solvedim, n=256):
    """The benchmark distribution with a_0 = c_{n-1} = 0 along the solve axis."""
    rng = np.random.default_rng(seed)
    a, b, c, d = rand_coeffs(rng, n ** 3, dtype)
    shp = (n, n, n)  # C order: the last axis is dims[0]
    ax = 2 - solvedim
    A, C = a.reshape(shp), c.reshape(shp)
    idx0 = [slice(None)] * 3
    idxn = [slice(None)] * 3
    idx0[ax], idxn[ax] = 0, n - 1
    A[tuple(idx0)] = 0
    C[tuple(idxn)] = 0
    return a, b, c, d


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_cube_256_against_reference_cpu(dtype, solvedim):
    dims = [256, 256, 256]
    a, b, c, d = cube_inputs(2560 + solvedim, dtype, solvedim)
    expect = oracle.ref_mtsv(a, b, c, d, solvedim=solvedim, dims=dims)
    td = dev(d)
    fn = tb.tridDmtsvStridedBatch if dtype == np.float64 else tb.tridSmtsvStridedBatch
    assert fn(dev(a), dev(b), dev(c), td, None, 3, solvedim, dims, dims) == 0
    got = host(td)
    err = rel_err(got, expect)
    assert err <= RTOL[dtype], err
    # sampled systems against FP64 dense LU
    rng = np.random.default_rng(7)
    pick = rng.choice(256 * 256, 64, replace=False)
    sys = [oracle.systems_view(x, dims, solvedim)[pick] for x in (a, b, c, d, got)]
    lu = oracle.dense_solve_systems(*(s.astype(np.float64) for s in sys[:4]))
    assert rel_err(sys[4], lu) <= RTOL[dtype]


@pytest.mark.parametrize("inc", [False, True])
def test_single_precision_padded_forms(inc):
    """tridSmtsvStridedBatchPadded[Inc]: every array with its own pads."""
    rng = np.random.default_rng(12 + inc)
    dims = [40, 33, 17]
    pads = {k: [40 + 2 * i, 33 + i, 17 + i] for i, k in enumerate("abcdu")}
    arrs = {}
    for k in "abcdu":
        n = int(np.prod(pads[k]))
        x = rng.uniform(-1, 1, n)
        if k == "b":
            x = 3.0 + rng.uniform(0, 1, n)
        arrs[k] = x.astype(np.float32)
    for solvedim in range(3):
        expect = oracle.mtsv(*(arrs[k] for k in "abcd"), arrs["u"], dims=dims, solvedim=solvedim,
                             inc=inc, array_pads=tuple(pads[k] for k in "abcdu"))
        t = {k: dev(arrs[k]) for k in "abcdu"}
        fn = tb.tridSmtsvStridedBatchPaddedInc if inc else tb.tridSmtsvStridedBatchPadded
        st = fn(t["a"], pads["a"], t["b"], pads["b"], t["c"], pads["c"], t["d"], pads["d"],
                t["u"], pads["u"], 3, solvedim, dims, opts=[0, 0, 0], sync=1)
        assert st == 0
        got = host(t["u"] if inc else t["d"])
        untouched = host(t["d"] if inc else t["u"])
        assert np.array_equal(untouched, arrs["d"] if inc else arrs["u"])
        assert rel_err(got, expect) <= 1e-5, solvedim


def block_batch(N, P, M, seed):
    """The block benchmark distribution, drawn on the GPU: off-diagonal
    entries U(-1,1)/M, diagonal blocks U(-1,1)/M + (2+U(0,1)) I, RHS N(0,1);
    interleaved layout (N, P, M, M)."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    kw = dict(device="cuda", dtype=torch.float64, generator=g)
    A = (torch.rand(N, P, M, M, **kw) * 2 - 1) / M
    C = (torch.rand(N, P, M, M, **kw) * 2 - 1) / M
    B = (torch.rand(N, P, M, M, **kw) * 2 - 1) / M
    B += (2 + torch.rand(N, P, 1, 1, **kw)) * torch.eye(M, device="cuda", dtype=torch.float64)
    d = torch.randn(N, P, M, **kw)
    return A, B, C, d


@pytest.mark.parametrize("M", [2, 4, 8])
def test_block_full_batch(M):
    N, P = 256, 32768
    A, B, C, d = block_batch(N, P, M, seed=M)
    x = block.btsv(A, B, C, d)
    w = torch.randn(N, P, M, device="cuda", dtype=torch.float64,
                    generator=torch.Generator(device="cuda").manual_seed(100 + M))
    dA, dB, dC, dd = block.btsv_adjoint(A, B, C, x, w)
    torch.cuda.synchronize()
    pick = torch.from_numpy(np.random.default_rng(M).choice(P, 256, replace=False)).cuda()
    hs = [t.index_select(1, pick).contiguous().cpu().numpy()
          for t in (A, B, C, d, x, w, dA, dB, dC, dd)]
    sA, sB, sC, sd, sx, sw, gA, gB, gC, gd = hs
    S = pick.numel()
    u = oracle.btsv(sA, sB, sC, sd, N, S, M, layout=0).reshape(N, S, M)
    assert rel_err(sx, u) <= 1e-12
    g = oracle.btsv(sA, sB, sC, sw, N, S, M, layout=0, transpose=True).reshape(N, S, M)
    assert rel_err(gd, g) <= 1e-12
    zero = np.zeros((1, S, M))
    assert rel_err(gA[1:], -np.einsum("npi,npj->npij", g, np.concatenate([zero, u[:-1]]))[1:]) <= 1e-12
    assert rel_err(gB, -np.einsum("npi,npj->npij", g, u)) <= 1e-12
    assert rel_err(gC[:-1], -np.einsum("npi,npj->npij", g, np.concatenate([u[1:], zero]))[:-1]) <= 1e-12


@needs_ref
def test_varlen_200k_against_reference_scalar():
    rng = np.random.default_rng(2024)
    nsys = 200_000
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(8192), nsys))).astype(np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    total = int(off[-1])
    g = torch.Generator(device="cuda").manual_seed(5)
    kw = dict(device="cuda", dtype=torch.float64, generator=g)
    a = torch.rand(total, **kw) * 2 - 1
    c = torch.rand(total, **kw) * 2 - 1
    b = a.abs() + c.abs() + 1 + torch.rand(total, **kw)
    d = torch.randn(total, **kw)
    d0 = d.clone()
    solve_varlen(a, b, c, d, torch.from_numpy(off).cuda())
    torch.cuda.synchronize()
    # the shortest, the longest and a random sample of systems
    pick = set(rng.choice(nsys, 300, replace=False).tolist())
    pick |= {int(np.argmin(lens)), int(np.argmax(lens)), 0, nsys - 1}
    for s in sorted(pick):
        lo, hi = int(off[s]), int(off[s + 1])
        sa, sb, sc, sd = (t[lo:hi].cpu().numpy() for t in (a, b, c, d0))
        ref = oracle.ref_trid_scalar(sa, sb, sc, sd, hi - lo, 1)
        got = d[lo:hi].cpu().numpy()
        assert rel_err(got, ref) <= 1e-12, (s, hi - lo)
