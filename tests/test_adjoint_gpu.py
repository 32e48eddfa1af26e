"""Adjoint and long-system parity (GPU, through the C ABI).

* the adjoint entry points (tridDmtsvStridedBatchAdjoint /
  tridSmtsvStridedBatchAdjoint) against the oracle's transposed Thomas
  (oracle/trid_oracle.c, oracle_adjoint_f64) for every axis and length class;
* the autograd Function against central finite differences (h = 1e-6) on
  sampled entries and against autograd through dense torch.linalg.solve;
* systems longer than one register-resident block (n > 512: block reduction,
  recursive block solve, block finish) against the oracle.
Bars: FP64 solves within 1e-12 and FP32 within 1e-5 relative max-norm;
gradients within 1e-12 of the transposed-Thomas oracle and 1e-10 of dense
autograd, finite differences within 1e-8 absolute for gradients of order
one (the FD rounding floor at h = 1e-6 and FP64 is ~1e-9).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import RTOL, dev, host, rand_coeffs, rel_err  # noqa: E402


@pytest.fixture(autouse=True)
def _auto_method():
    tb.set_method(0)
    yield
    tb.set_method(0)


def strided_systems(x, dims, solvedim):
    return oracle.systems_view(x, dims, solvedim)


def expected_adjoint(a, b, c, u, w, dims, solvedim):
    """Oracle gradients in the arrays' own layout."""
    sv = lambda v: np.ascontiguousarray(strided_systems(v, dims, solvedim))
    n = dims[solvedim]
    g, ga, gb, gc = oracle.adjoint(sv(a), sv(b), sv(c), sv(u), sv(w), n)
    out = []
    for arr in (ga, gb, gc, g):
        full = np.zeros(int(np.prod(dims)))
        view = full.reshape(dims[::-1])
        ax = len(dims) - 1 - solvedim
        moved = np.moveaxis(view, ax, -1)
        moved[...] = arr.reshape(moved.shape)
        out.append(full)
    return out  # da, db, dc, dd


def run_adjoint(dtype, dims, solvedim, seed=0, method=None):
    rng = np.random.default_rng(seed)
    size = int(np.prod(dims))
    a, b, c, d = rand_coeffs(rng, size, np.float64)
    w = rng.standard_normal(size)
    u = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
    exp = expected_adjoint(a, b, c, u, w, dims, solvedim)
    if method is not None:
        tb.set_method(*method)
    t = [dev(x.astype(dtype)) for x in (a, b, c, u, w)]
    outs = [torch.full_like(t[0], np.nan) for _ in range(4)]
    fn = tb.tridDmtsvStridedBatchAdjoint if dtype == np.float64 else tb.tridSmtsvStridedBatchAdjoint
    st = fn(*t, *outs, len(dims), solvedim, dims, dims)
    assert st == 0
    tol = 1e-12 if dtype == np.float64 else 2e-5
    for got, want in zip(outs, exp):
        assert rel_err(host(got), want) <= tol


@pytest.mark.parametrize("n", [1, 2, 7, 64, 256, 300, 512, 1024, 5000, 8192])
def test_adjoint_axis0(n):
    run_adjoint(np.float64, [n, 23], 0, seed=n)


@pytest.mark.parametrize("n", [3, 100, 256, 700])
@pytest.mark.parametrize("solvedim", [1, 2])
def test_adjoint_strided(n, solvedim):
    dims = [20, n, 3] if solvedim == 1 else [20, 3, n]
    run_adjoint(np.float64, dims, solvedim, seed=n + solvedim)


def test_adjoint_fp32():
    run_adjoint(np.float32, [256, 40], 0, seed=5)
    run_adjoint(np.float32, [40, 256], 1, seed=6)


@pytest.mark.parametrize("method", [(2, 16, 0), (3, 4, 4), (3, 8, 16)])
def test_adjoint_methods(method):
    run_adjoint(np.float64, [33, 600, 2], 1, seed=9, method=method)


def test_adjoint_null_outputs_and_dd_aliasing_w():
    rng = np.random.default_rng(4)
    dims = [128, 17]
    a, b, c, d = rand_coeffs(rng, 128 * 17)
    w = rng.standard_normal(128 * 17)
    u = oracle.mtsv(a, b, c, d, dims=dims, solvedim=0)
    _, _, _, dd = expected_adjoint(a, b, c, u, w, dims, 0)
    t = [dev(x) for x in (a, b, c, u)]
    tw = dev(w)
    st = tb.tridDmtsvStridedBatchAdjoint(*t, tw, None, None, None, tw, 2, 0, dims, dims)
    assert st == 0
    assert rel_err(host(tw), dd) <= 1e-12


# ------------------------------------------------------------ autograd --
def test_autograd_against_dense_linalg_solve():
    """32 systems of n=1024, FP64: loss = sum(w*u)."""
    torch.manual_seed(0)
    S, n = 32, 1024
    a = (torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1)
    c = (torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1)
    b = a.abs() + c.abs() + 1 + torch.rand(S, n, dtype=torch.float64, device="cuda")
    d = torch.randn(S, n, dtype=torch.float64, device="cuda")
    w = torch.randn(S, n, dtype=torch.float64, device="cuda")
    leaves = [x.clone().requires_grad_(True) for x in (a, b, c, d)]
    u = tb.trid_solve(*leaves, dim=-1)
    (u * w).sum().backward()
    ours = [x.grad for x in leaves]

    ref = [x.clone().requires_grad_(True) for x in (a, b, c, d)]
    A = torch.diag_embed(ref[1]) + torch.diag_embed(ref[0][:, 1:], -1) + \
        torch.diag_embed(ref[2][:, :-1], 1)
    ud = torch.linalg.solve(A, ref[3].unsqueeze(-1)).squeeze(-1)
    (ud * w).sum().backward()
    assert rel_err(u.detach().cpu().numpy(), ud.detach().cpu().numpy()) <= 1e-12
    for g1, g2 in zip(ours, ref):
        err = (g1 - g2.grad).abs().max() / g2.grad.abs().max()
        assert err <= 1e-10, float(err)


def test_autograd_finite_differences():
    """Central differences, h = 1e-6, on 64 sampled entries of a, b, c, d."""
    torch.manual_seed(1)
    S, n = 64, 1024
    a = (torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1)
    c = (torch.rand(S, n, dtype=torch.float64, device="cuda") * 2 - 1)
    b = a.abs() + c.abs() + 1 + torch.rand(S, n, dtype=torch.float64, device="cuda")
    d = torch.randn(S, n, dtype=torch.float64, device="cuda")
    w = torch.randn(S, n, dtype=torch.float64, device="cuda")
    leaves = [x.clone().requires_grad_(True) for x in (a, b, c, d)]
    u = tb.trid_solve(*leaves, dim=-1)
    (u * w).sum().backward()
    rng = np.random.default_rng(2)
    h = 1e-6
    errs, gmax = [], 0.0
    for k in range(64):
        which = k % 4
        s = int(rng.integers(S))
        i = int(rng.integers(1, n - 1))
        base = [x.detach().clone() for x in (a, b, c, d)]
        plus = [x.clone() for x in base]
        minus = [x.clone() for x in base]
        plus[which][s, i] += h
        minus[which][s, i] -= h
        up = tb.trid_solve(*plus, dim=-1)
        um = tb.trid_solve(*minus, dim=-1)
        fd = float(((up - um)[s] * w[s]).sum() / (2 * h))
        g = float(leaves[which].grad[s, i])
        errs.append(abs(fd - g))
        gmax = max(gmax, abs(g))
    # gradient error <= 1e-8 against finite differences, relative to the
    # largest sampled gradient (the FD rounding floor at h = 1e-6 is ~1e-9
    # absolute: eps * sqrt(n) * |w| * |u| / (2h))
    assert max(errs) <= 1e-8 * max(1.0, gmax), (max(errs), gmax)


# --------------------------------------------------------- long systems --
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [513, 1000, 1024, 4097, 8192, 20000])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("method", [None, (3, 8, 0)])
def test_long_axis0(dtype, n, inc, method):
    """8192 rows: whole 256-row blocks (the guard-free block kernels); method 3
    takes the blocked partition from 513 rows on (no one-CTA kernel)."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(n), dtype, [n, 9], 0, inc=inc, method=method)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [257, 300, 384, 385, 700, 768, 1100, 1152, 1153, 1536, 2048, 2500,
                               3000, 3072, 3073, 4000, 4096])
@pytest.mark.parametrize("inc", [False, True])
def test_one_cta_row_layouts(dtype, n, inc):
    """Axis-0 systems solved whole by one CTA: 12 rows per lane where that
    pads fewer rows (257..384, 513..768, 1025..1152), 16 otherwise, with the
    register-capped variants for 3..6 warps (1025..3072 rows) and the
    uncapped ones past them; pads[0] = n + 3 keeps the rows off the TMA grid."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(n + inc), dtype, [n, 23], 0, pads=[n + 3, 23], inc=inc)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n,nsys", [(4097, 400), (5000, 300), (65536, 20), (65535, 19)])
@pytest.mark.parametrize("inc", [False, True])
def test_long_axis0_many_steps(dtype, n, nsys, inc):
    """Batches of long systems whose block rows span many CTAs (the reduce
    and finish launches of the blocked partition and the block system solved
    as its own batch), ragged last blocks included."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(n + nsys), dtype, [n, nsys], 0, inc=inc)


@pytest.mark.parametrize("inc", [False, True])
def test_long_axis0_padded_outer(inc):
    """Padded outer axes (3-D arrays) on the blocked partition."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(7), np.float64, [6000, 5, 3], 0, pads=[6000, 7, 4], inc=inc)


@pytest.mark.parametrize("n", [600, 2000])
@pytest.mark.parametrize("solvedim", [1, 2])
@pytest.mark.parametrize("method", [None, (3, 16, 4), (2, 8, 16)])
def test_long_strided(n, solvedim, method):
    from test_scalar_gpu import run_case
    dims = [24, n, 3] if solvedim == 1 else [24, 3, n]
    run_case(np.random.default_rng(n + solvedim), np.float64, dims, solvedim, method=method)


def test_long_65536_batch():
    """The long-system configuration's length (n = 65,536), 16 systems."""
    from test_scalar_gpu import run_case
    run_case(np.random.default_rng(65536), np.float64, [65536, 16], 0)


@pytest.mark.parametrize("n", [1500, 9000])
def test_long_padded_per_array(n):
    rng = np.random.default_rng(12)
    dims = [n, 5]
    pads = {k: [n + 3 * i, 5] for i, k in enumerate("abcdu")}
    arrs = {}
    for k in "abcdu":
        nn = int(np.prod(pads[k]))
        arrs[k] = 3.0 + rng.uniform(0, 1, nn) if k == "b" else rng.uniform(-1, 1, nn)
    ap = tuple(pads[k] for k in "abcdu")
    expect = oracle.mtsv(*(arrs[k] for k in "abcd"), dims=dims, solvedim=0, array_pads=ap)
    t = {k: dev(arrs[k]) for k in "abcdu"}
    st = tb.tridDmtsvStridedBatchPadded(t["a"], pads["a"], t["b"], pads["b"], t["c"], pads["c"],
                                        t["d"], pads["d"], t["u"], pads["u"], 2, 0, dims, sync=1)
    assert st == 0
    assert rel_err(host(t["d"]), expect) <= RTOL[np.float64]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim", [([32, 50], 0), ([300, 21], 0), ([1024, 9], 0),
                                           ([5000, 3], 0), ([40, 129, 3], 1), ([24, 5, 70], 2)])
def test_out_of_place_solve(dtype, dims, solvedim):
    """tridX mtsvStridedBatchOut: x = A^{-1} d written next to d, d intact."""
    rng = np.random.default_rng(sum(dims) + solvedim)
    size = int(np.prod(dims))
    a, b, c, d = rand_coeffs(rng, size, dtype)
    expect = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
    td = dev(d)
    x = torch.full_like(td, float("nan"))
    fn = tb.tridDmtsvStridedBatchOut if dtype == np.float64 else tb.tridSmtsvStridedBatchOut
    assert fn(dev(a), dev(b), dev(c), td, x, len(dims), solvedim, dims, dims) == 0
    assert np.array_equal(host(td), d)
    assert rel_err(host(x), expect) <= (1e-12 if dtype == np.float64 else 1e-5)
    # x may be d: the in-place solve
    assert fn(dev(a), dev(b), dev(c), td, td, len(dims), solvedim, dims, dims) == 0
    assert rel_err(host(td), expect) <= (1e-12 if dtype == np.float64 else 1e-5)
