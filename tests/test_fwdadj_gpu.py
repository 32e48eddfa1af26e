"""Forward solve + adjoint in one call (GPU, through the C ABI):
tridDmtsvStridedBatchFwdAdj / tridSmtsvStridedBatchFwdAdj against the oracle's
forward solve (oracle_mtsv_f64, pinned to the reference's CPU path) and its
transposed-Thomas adjoint (oracle_adjoint_f64).  Covers the one-kernel path
(unit-stride axis up to 4096 rows), the short systems under it, and the
two-pass fallback (strided axes, n > 4096).  Also the one-CTA forward and
separate-adjoint kernels that serve tridDmtsvStridedBatch and
tridDmtsvStridedBatchAdjoint at those lengths.
Bars: FP64 1e-12 and FP32 2e-5 relative max-norm."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import dev, host, rand_coeffs, rel_err  # noqa: E402
from test_adjoint_gpu import expected_adjoint  # noqa: E402


@pytest.fixture(autouse=True)
def _auto_method():
    tb.set_method(0)
    yield
    tb.set_method(0)


def run_fused(dtype, dims, solvedim, seed=0, alias=False, nulls=()):
    rng = np.random.default_rng(seed)
    size = int(np.prod(dims))
    a, b, c, d = rand_coeffs(rng, size, np.float64)
    w = rng.standard_normal(size)
    # the oracle solves the same (rounded) system in FP64
    a, b, c, d, w = (v.astype(dtype).astype(np.float64) for v in (a, b, c, d, w))
    x = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
    exp = expected_adjoint(a, b, c, x, w, dims, solvedim)  # da, db, dc, dd
    t = [dev(v.astype(dtype)) for v in (a, b, c, d, w)]
    tx = t[3] if alias else torch.full_like(t[0], np.nan)
    outs = [None if k in nulls else (t[4] if alias and k == 3 else torch.full_like(t[0], np.nan))
            for k in range(4)]
    fn = (tb.tridDmtsvStridedBatchFwdAdj if dtype == np.float64
          else tb.tridSmtsvStridedBatchFwdAdj)
    st = fn(*t, tx, *outs, len(dims), solvedim, dims, dims)
    assert st == 0
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert rel_err(host(tx), x) <= tol
    for k, (got, want) in enumerate(zip(outs, exp)):
        if got is not None:
            assert rel_err(host(got), want) <= tol, k


@pytest.mark.parametrize("n", [513, 700, 1024, 1500, 2048, 2049, 3000, 4096])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_fused_one_kernel(n, dtype):
    run_fused(dtype, [n, 7], 0, seed=n)


@pytest.mark.parametrize("method", [(6, 4), (6, 8), (6, 16)])
@pytest.mark.parametrize("n", [65, 66, 100, 257, 511, 1000, 1024, 1025, 2500, 4096])
def test_fused_forced_kernel(method, n):
    tb.set_method(*method)
    run_fused(np.float64, [n, 5], 0, seed=n + method[1])
    run_fused(np.float32, [n, 3], 0, seed=n + method[1] + 1)


@pytest.mark.parametrize("n", [1, 2, 31, 256, 512])
def test_fused_short(n):
    run_fused(np.float64, [n, 11], 0, seed=n)


@pytest.mark.parametrize("dims,solvedim", [([20, 300, 3], 1), ([6, 5, 700], 2),
                                           ([5000, 3], 0), ([1024, 4, 3], 1)])
def test_fused_two_pass(dims, solvedim):
    run_fused(np.float64, dims, solvedim, seed=sum(dims))


def test_fused_aliasing_and_null_outputs():
    run_fused(np.float64, [1024, 9], 0, seed=1, alias=True)
    run_fused(np.float64, [1024, 9], 0, seed=2, nulls=(0, 2))
    run_fused(np.float64, [300, 9, 2], 1, seed=3, alias=True, nulls=(1,))


def test_fused_padded_rows():
    # rows padded to 1030 elements: the systems start off 8-element boundaries
    rng = np.random.default_rng(4)
    n, S, pad = 1000, 6, 1030
    dims, pads = [n, S], [pad, S]
    a, b, c, d = rand_coeffs(rng, pad * S)
    w = rng.standard_normal(pad * S)
    sv = lambda v: np.ascontiguousarray(v.reshape(S, pad)[:, :n])
    x = oracle.mtsv(sv(a), sv(b), sv(c), sv(d), dims=dims, solvedim=0).ravel()
    g, ga, gb, gc = oracle.adjoint(sv(a), sv(b), sv(c), x, sv(w), n)
    t = [dev(v) for v in (a, b, c, d, w)]
    tx = torch.zeros_like(t[0])
    outs = [torch.zeros_like(t[0]) for _ in range(4)]
    assert tb.tridDmtsvStridedBatchFwdAdj(*t, tx, *outs, 2, 0, dims, pads) == 0
    cut = lambda v: host(v).reshape(S, pad)[:, :n].ravel()
    assert rel_err(cut(tx), x) <= 1e-12
    for got, want in zip(outs, (ga, gb, gc, g)):
        assert rel_err(cut(got), want.ravel()) <= 1e-12


def test_solve_fwd_adj_torch_matches_autograd():
    torch.manual_seed(7)
    S, n = 64, 1024
    a = torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1
    c = torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1
    b = a.abs() + c.abs() + 1 + torch.rand(S, n, dtype=torch.float64, device="cuda")
    d = torch.randn(S, n, dtype=torch.float64, device="cuda")
    w = torch.randn(S, n, dtype=torch.float64, device="cuda")
    x, grads = tb.solve_fwd_adj(a, b, c, d, w)
    leaves = [v.clone().requires_grad_(True) for v in (a, b, c, d)]
    u = tb.trid_solve(*leaves)
    (u * w).sum().backward()
    assert rel_err(host(x), host(u.detach())) <= 1e-13
    for g1, leaf in zip(grads, leaves):
        assert rel_err(host(g1), host(leaf.grad)) <= 1e-12


@pytest.mark.parametrize("n", [600, 2048, 4000])
@pytest.mark.parametrize("inc", [False, True])
def test_one_kernel_forward_fp32(n, inc):
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(n + 1), np.float32, [n, 5], 0, inc=inc)


@pytest.mark.parametrize("n", [513, 2049, 4096])
def test_one_kernel_adjoint(n):
    from test_adjoint_gpu import run_adjoint
    run_adjoint(np.float64, [n, 6], 0, seed=n + 2)
    run_adjoint(np.float32, [n, 6], 0, seed=n + 3)


@pytest.mark.parametrize("method", [6])
@pytest.mark.parametrize("n", [65, 97, 300, 1024, 1031, 3000, 5000, 7000])
@pytest.mark.parametrize("inc", [False, True])
def test_forced_kernel_forward(method, n, inc):
    """Method 6 forced: where its limit excludes the system (past 4096
    rows) the call still returns the solution through another kernel."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(n + method), np.float64, [n, 4], 0, inc=inc,
             method=(method, 0, 0))


@pytest.mark.parametrize("method", [(6, 4), (6, 16)])
@pytest.mark.parametrize("n", [65, 300, 1024, 1031, 5000])
def test_forced_kernel_adjoint(method, n):
    from test_adjoint_gpu import run_adjoint
    run_adjoint(np.float64, [n, 4], 0, seed=n + method[1], method=(*method, 0))
