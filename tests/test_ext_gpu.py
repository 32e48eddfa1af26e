"""Complex and FP32-storage / FP64-arithmetic strided-batch solves (GPU,
through the C ABI).

Complex: tridC/ZmtsvStridedBatch[Inc] against the complex oracle (the real
Thomas restatement in C99 complex arithmetic, pinned to the real oracle and
to dense complex LU) on rows diagonally dominant in modulus.  Bars: complex128
1e-12, complex64 1e-5 (relative max-norm of the modulus).

Mixed: tridSmtsvStridedBatchMixed[Inc] against the FP64 oracle on the widened
inputs, rounded to float32 once (Inc: float32(float64(u) + x)).  Bar 2.5e-7
relative max-norm: two float32 units in the last place of the largest entry,
room for an FP64 result within 1e-15 of the oracle's to round the other way.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import rand_coeffs, rand_complex_coeffs, rel_err  # noqa: E402

CPLX = {
    "z": (np.complex128, tb.tridZmtsvStridedBatch, tb.tridZmtsvStridedBatchInc, 1e-12),
    "c": (np.complex64, tb.tridCmtsvStridedBatch, tb.tridCmtsvStridedBatchInc, 1e-5),
}
MIXED_TOL = 2.5e-7


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def geometry(n, solvedim, rows16=False):
    """dims with n along solvedim; padded axes 0 and 2.  rows16: axis 0 of 48
    systems padded to 52 (whole 16-system tiles, rows on 16-byte boundaries:
    the strided axes take 16-byte copies)."""
    dims = [48 if rows16 else 37, 5, 3]
    dims[solvedim] = n
    pads = [dims[0] + (4 if rows16 else 2), dims[1], dims[2] + 1]
    return dims, pads


def outside(dims, pads):
    mask = np.ones(pads[::-1], dtype=bool)
    mask[:dims[2], :dims[1], :dims[0]] = False
    return mask.ravel()


@pytest.mark.parametrize("kind", ["z", "c"])
@pytest.mark.parametrize("n", [1, 2, 3, 31, 64, 129, 256, 300, 512, 700])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("rows16", [False, True])
def test_complex_strided(kind, n, solvedim, inc, rows16):
    if rows16 and solvedim == 0:
        pytest.skip("axis 0 has no tiles of systems")
    ndt, f, finc, tol = CPLX[kind]
    rng = np.random.default_rng(1000 * n + 10 * solvedim + inc + (7 if kind == "c" else 0))
    dims, pads = geometry(n, solvedim, rows16)
    size = int(np.prod(pads))
    a, b, c, d = rand_complex_coeffs(rng, size, ndt)
    u = (rng.standard_normal(size) + 1j * rng.standard_normal(size)).astype(ndt)
    expect = oracle.mtsv(a, b, c, d, u=u if inc else None, dims=dims, pads=pads,
                         solvedim=solvedim, inc=inc)
    A, B, C, D, U = (dev(v) for v in (a, b, c, d, u))
    st = (finc if inc else f)(A, B, C, D, U if inc else None, 3, solvedim, dims, pads)
    assert st == 0
    out = (U if inc else D).cpu().numpy()
    sv = lambda v: oracle.systems_view(v, dims, solvedim, pads)
    assert rel_err(sv(out), sv(expect)) <= tol
    m = outside(dims, pads)
    assert np.array_equal(out[m], (u if inc else d)[m])  # padding untouched
    if inc:
        assert np.array_equal(D.cpu().numpy(), d)  # Inc leaves d unchanged


@pytest.mark.parametrize("n", [1, 2, 5, 64, 200, 256, 400, 512, 1000])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("rows16", [False, True])
def test_mixed_strided(n, solvedim, inc, rows16):
    if rows16 and solvedim == 0:
        pytest.skip("axis 0 has no tiles of systems")
    rng = np.random.default_rng(77 * n + 3 * solvedim + inc)
    dims, pads = geometry(n, solvedim, rows16)
    size = int(np.prod(pads))
    a, b, c, d = rand_coeffs(rng, size, np.float32)
    u = rng.standard_normal(size).astype(np.float32)
    w = [v.astype(np.float64) for v in (a, b, c, d, u)]
    e64 = oracle.mtsv(*w[:4], u=w[4] if inc else None, dims=dims, pads=pads, solvedim=solvedim,
                      inc=inc)
    expect = e64.astype(np.float32)
    A, B, C, D, U = (dev(v) for v in (a, b, c, d, u))
    fn = tb.tridSmtsvStridedBatchMixedInc if inc else tb.tridSmtsvStridedBatchMixed
    assert fn(A, B, C, D, U if inc else None, 3, solvedim, dims, pads) == 0
    out = (U if inc else D).cpu().numpy()
    sv = lambda v: oracle.systems_view(v, dims, solvedim, pads)
    assert rel_err(sv(out), sv(expect)) <= MIXED_TOL
    m = outside(dims, pads)
    assert np.array_equal(out[m], (u if inc else d)[m])


def test_mixed_beats_fp32_arithmetic():
    """On 1024-row systems the FP64-arithmetic result sits within rounding
    of the FP64 solution, closer than the FP32-arithmetic solve."""
    rng = np.random.default_rng(9)
    shape = (64, 1024)
    a, b, c, d = rand_coeffs(rng, shape, np.float32)
    e64 = oracle.mtsv(*(v.astype(np.float64).ravel() for v in (a, b, c, d)), dims=[1024, 64],
                      solvedim=0).reshape(shape)
    xm = tb.solve(dev(a), dev(b), dev(c), dev(d), fp64_arithmetic=True).cpu().numpy()
    x32 = tb.solve(dev(a), dev(b), dev(c), dev(d)).cpu().numpy()
    em, e32 = rel_err(xm, e64), rel_err(x32, e64)
    assert em <= 1e-7
    assert em < e32


@pytest.mark.parametrize("kind", ["z", "c", "mixed"])
def test_first_a_and_last_c_never_read(kind):
    rng = np.random.default_rng(4)
    n, nsys = 100, 40
    if kind == "mixed":
        a, b, c, d = rand_coeffs(rng, (nsys, n), np.float32)
        tol = MIXED_TOL
    else:
        a, b, c, d = rand_complex_coeffs(rng, (nsys, n), CPLX[kind][0])
        tol = CPLX[kind][3]
    if kind == "mixed":
        expect = oracle.mtsv(*(v.astype(np.float64).ravel() for v in (a, b, c, d)),
                             dims=[n, nsys], solvedim=0).astype(np.float32)
    else:
        expect = oracle.mtsv(a.ravel(), b.ravel(), c.ravel(), d.ravel(), dims=[n, nsys],
                             solvedim=0)
    a2, c2 = a.copy(), c.copy()
    a2[:, 0] = np.nan
    c2[:, -1] = np.inf
    for layout in ("rows", "columns"):
        if layout == "rows":
            x = tb.solve(dev(a2), dev(b), dev(c2), dev(d), dim=-1,
                         fp64_arithmetic=kind == "mixed").cpu().numpy()
            assert rel_err(x.ravel(), expect) <= tol
        else:  # the same systems along the strided axis
            t = lambda v: dev(np.ascontiguousarray(v.T))
            x = tb.solve(t(a2), t(b), t(c2), t(d), dim=0,
                         fp64_arithmetic=kind == "mixed").cpu().numpy()
            assert rel_err(x.T.ravel(), expect) <= tol


def test_complex_through_solve_matches_dense():
    rng = np.random.default_rng(12)
    a, b, c, d = rand_complex_coeffs(rng, (8, 50), np.complex128)
    x = tb.solve(dev(a), dev(b), dev(c), dev(d.copy())).cpu().numpy()
    xd = oracle.dense_solve_systems(a, b, c, d)
    assert rel_err(x, xd) <= 1e-12


def test_unsupported_dtype_and_flag_rejected():
    x = torch.ones(4, 8, dtype=torch.float16, device="cuda")
    with pytest.raises(TypeError):
        tb.solve(x, x, x, x)
    y = torch.ones(4, 8, dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError):
        tb.solve(y, y, y, y, fp64_arithmetic=True)
