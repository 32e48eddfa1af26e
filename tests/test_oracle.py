"""Pin the CPU oracle (test infrastructure) before trusting it.

* every golden fixture of the reference's file-driven tests
  (scalar/test/test_cpu.cpp:88-252, scalar/test/test_cuda.cu:58-137), with the
  reference's tolerances (scalar/test/utils.hpp:14-17, test_cpu.cpp:10-32);
* the reference's own CPU library compiled unmodified (oracle/_ref), on the
  same seeded inputs, including Inc and padded arrays;
* an FP64 dense-LU oracle for the block solver and the adjoint, which have
  no reference golden vectors;
* the reference's sequential ADI gold program (apps/adi/src/adi_orig.c).
"""

import glob
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))

ABS_TOL = {np.float64: 1e-11, np.float32: 1e-6}   # utils.hpp:14-17
REL_TOL = {np.float64: 1e-11, np.float32: 1e-5}

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference CPU code not built (make -C oracle ref)")


def require_allclose(expected, actual, dtype):
    """test_cpu.cpp:10-32: |e-a| <= abs + rel*min(|e|,|a|) elementwise."""
    e = np.asarray(expected, dtype=np.float64)
    a = np.asarray(actual, dtype=np.float64)
    tol = ABS_TOL[dtype] + REL_TOL[dtype] * np.minimum(np.abs(e), np.abs(a))
    bad = np.abs(e - a) > tol
    assert not bad.any(), f"{bad.sum()} mismatches, max diff {np.abs(e - a).max()}"


def load(path, dtype):
    z = np.load(path)
    dims = [int(v) for v in z["dims"]]
    arrs = [z[k].astype(dtype) for k in "abcd"]
    expect = z["u"] if dtype == np.float64 else z["u_float"]
    return dims, int(z["solvedim"]), arrs, expect


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_matches_golden(path, dtype):
    if dtype == np.float32 and "reduced" in path:
        pytest.skip("the reference checks this fixture in FP64 only (test_cuda_mpi.cu:289-291)")
    dims, solvedim, (a, b, c, d), expect = load(path, dtype)
    out = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
    require_allclose(expect, out, dtype)


@needs_ref
@pytest.mark.parametrize("path", [p for p in GOLDEN if "four_dim" not in p],
                         ids=[os.path.basename(p)[:-4] for p in GOLDEN if "four_dim" not in p])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_reference_cpu_matches_golden(path, dtype):
    if dtype == np.float32 and "reduced" in path:
        pytest.skip("the reference checks this fixture in FP64 only (test_cuda_mpi.cu:289-291)")
    dims, solvedim, (a, b, c, d), expect = load(path, dtype)
    simd = 4 if dtype == np.float64 else 8
    if solvedim > 0 and dims[0] % simd:
        pytest.skip("reference y/z path needs dims[0] % SIMD_VEC == 0 (test_cpu.cpp:178-183)")
    out = oracle.ref_mtsv(a, b, c, d, solvedim=solvedim, dims=dims)
    require_allclose(expect, out, dtype)


def rand_system(rng, shape, dtype):
    """Strictly diagonally dominant coefficients (the benchmark distribution)."""
    a = rng.uniform(-1, 1, shape)
    c = rng.uniform(-1, 1, shape)
    b = np.abs(a) + np.abs(c) + rng.uniform(1, 2, shape)
    d = rng.standard_normal(shape)
    u = rng.standard_normal(shape)
    return [x.astype(dtype) for x in (a, b, c, d, u)]


@needs_ref
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
def test_oracle_matches_reference_cpu(dtype, solvedim, inc):
    rng = np.random.default_rng(100 + solvedim)
    dims = [24, 20, 12]
    pads = [32, 22, 13]          # padded arrays, pads[0] % SIMD width == 0
    size = int(np.prod(pads))
    a, b, c, d, u = rand_system(rng, size, dtype)
    ours = oracle.mtsv(a, b, c, d, u, dims=dims, pads=pads, solvedim=solvedim, inc=inc)
    ref = oracle.ref_mtsv(a, b, c, d, u, dims=dims, pads=pads, solvedim=solvedim, inc=inc)
    # same algorithm, same operation order: only FMA contraction in the
    # reference's -O3 -mfma build can differ.
    tol = 1e-13 if dtype == np.float64 else 2e-5
    scale = np.abs(ref).max()
    assert np.abs(ours - ref).max() <= tol * scale
    if inc:
        # Inc leaves d unmodified and only touches u inside dims
        mask = np.zeros(pads[::-1], dtype=bool)
        mask[:dims[2], :dims[1], :dims[0]] = True
        assert np.array_equal(ours.reshape(pads[::-1])[~mask], u.reshape(pads[::-1])[~mask])


def test_oracle_against_dense_lu():
    rng = np.random.default_rng(7)
    dims = [17, 9, 5]
    for solvedim in range(3):
        a, b, c, d, _ = rand_system(rng, int(np.prod(dims)), np.float64)
        x = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
        sv = lambda v: oracle.systems_view(v, dims, solvedim)
        xd = oracle.dense_solve_systems(sv(a), sv(b), sv(c), sv(d))
        assert np.abs(sv(x) - xd).max() / np.abs(xd).max() < 1e-13


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-13), (np.complex64, 2e-5)])
def test_complex_oracle_against_dense_lu(dtype, tol):
    """The complex restatement (same Thomas in complex arithmetic) against
    dense complex LU on every axis, with pads."""
    from helpers import rand_complex_coeffs
    rng = np.random.default_rng(17)
    dims, pads = [13, 6, 4], [15, 6, 5]
    for solvedim in range(3):
        a, b, c, d = rand_complex_coeffs(rng, int(np.prod(pads)), dtype)
        x = oracle.mtsv(a, b, c, d, dims=dims, pads=pads, solvedim=solvedim)
        sv = lambda v: oracle.systems_view(v, dims, solvedim, pads)
        xd = oracle.dense_solve_systems(sv(a), sv(b), sv(c), sv(d))
        assert np.abs(sv(x) - xd).max() / np.abs(xd).max() < tol
        u = (rng.standard_normal(a.size) + 1j * rng.standard_normal(a.size)).astype(dtype)
        ui = oracle.mtsv(a, b, c, d, u=u, dims=dims, pads=pads, solvedim=solvedim, inc=True)
        assert np.abs(sv(ui) - sv(u) - xd).max() / np.abs(xd).max() < 2 * tol


@pytest.mark.parametrize("rdt,cdt", [(np.float64, np.complex128), (np.float32, np.complex64)])
def test_complex_oracle_reduces_to_real_oracle(rdt, cdt):
    """With zero imaginary parts the complex restatement gives the real one's
    answer (which the golden fixtures and the reference CPU build pin)."""
    rng = np.random.default_rng(5)
    dims = [40, 7, 3]
    a, b, c, d, _ = rand_system(rng, int(np.prod(dims)), rdt)
    tol = 1e-15 if rdt == np.float64 else 1e-6
    for solvedim in range(3):
        xr = oracle.mtsv(a, b, c, d, dims=dims, solvedim=solvedim)
        xc = oracle.mtsv(*(v.astype(cdt) for v in (a, b, c, d)), dims=dims, solvedim=solvedim)
        assert np.abs(xc.imag).max() == 0
        assert np.abs(xc.real - xr).max() / np.abs(xr).max() <= tol


def test_oracle_ignores_a0_and_cn():
    """a[0] and c[n-1] of every system are never read (trid_cpu.cpp:360-401)."""
    rng = np.random.default_rng(3)
    a, b, c, d, _ = rand_system(rng, (6, 40), np.float64)
    x1 = oracle.mtsv(a.ravel(), b.ravel(), c.ravel(), d.ravel(), dims=[40, 6], solvedim=0)
    a2, c2 = a.copy(), c.copy()
    a2[:, 0] = 1e300
    c2[:, -1] = np.nan
    x2 = oracle.mtsv(a2.ravel(), b.ravel(), c2.ravel(), d.ravel(), dims=[40, 6], solvedim=0)
    assert np.array_equal(x1, x2)


def test_oracle_ndim_up_to_8():
    rng = np.random.default_rng(11)
    dims = [3, 2, 4, 2, 3, 2, 2, 5]
    pads = [4, 2, 5, 2, 3, 3, 2, 5]
    size = int(np.prod(pads))
    a, b, c, d, _ = rand_system(rng, size, np.float64)
    for solvedim in (0, 3, 7):
        x = oracle.mtsv(a, b, c, d, dims=dims, pads=pads, solvedim=solvedim)
        sv = lambda v: oracle.systems_view(v, dims, solvedim, pads)
        xd = oracle.dense_solve_systems(sv(a), sv(b), sv(c), sv(d))
        assert np.abs(sv(x) - xd).max() < 1e-13


@needs_ref
def test_varlen_oracle_matches_reference_scalar():
    rng = np.random.default_rng(5)
    lens = rng.integers(1, 300, 40)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    a, b, c, d, _ = rand_system(rng, int(off[-1]), np.float64)
    x = oracle.varlen(a, b, c, d, off)
    for s in range(len(lens)):
        o, n = off[s], lens[s]
        ref = oracle.ref_trid_scalar(a[o:o + n], b[o:o + n], c[o:o + n], d[o:o + n], n, 1)
        assert np.abs(x[o:o + n] - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_adjoint_oracle_against_dense():
    rng = np.random.default_rng(9)
    n, S = 33, 5
    a, b, c, d, w = rand_system(rng, (S, n), np.float64)
    u = oracle.dense_solve_systems(a, b, c, d)
    g, ga, gb, gc = (x.reshape(S, n) for x in oracle.adjoint(a, b, c, u, w, n))
    for s in range(S):
        A = np.diag(b[s]) + np.diag(a[s, 1:], -1) + np.diag(c[s, :-1], 1)
        gd = np.linalg.solve(A.T, w[s])
        assert np.allclose(g[s], gd, rtol=1e-13, atol=1e-13)
        G = -np.outer(gd, u[s])            # dL/dA = -g u^T
        assert np.allclose(gb[s], np.diag(G), atol=1e-13)
        assert np.allclose(ga[s, 1:], np.diag(G, -1), atol=1e-13) and ga[s, 0] == 0
        assert np.allclose(gc[s, :-1], np.diag(G, 1), atol=1e-13) and gc[s, -1] == 0


def block_system(rng, N, P, M):
    A = rng.uniform(-1, 1, (N, P, M, M)) / M
    B = rng.uniform(-1, 1, (N, P, M, M)) / M + (2 + rng.uniform(0, 1, (N, P, 1, 1))) * np.eye(M)
    C = rng.uniform(-1, 1, (N, P, M, M)) / M
    d = rng.standard_normal((N, P, M))
    return A, B, C, d


def dense_block(A, B, C, d, p, transpose=False):
    N, P, M, _ = A.shape
    K = np.zeros((N * M, N * M))
    for n in range(N):
        K[n * M:(n + 1) * M, n * M:(n + 1) * M] = B[n, p]
        if n > 0:
            K[n * M:(n + 1) * M, (n - 1) * M:n * M] = A[n, p]
        if n < N - 1:
            K[n * M:(n + 1) * M, (n + 1) * M:(n + 2) * M] = C[n, p]
    if transpose:
        K = K.T
    return np.linalg.solve(K, d[:, p].reshape(-1)).reshape(N, M)


@pytest.mark.parametrize("M", [1, 2, 3, 4, 5, 8])
@pytest.mark.parametrize("transpose", [False, True])
def test_block_oracle_against_dense_lu(M, transpose):
    rng = np.random.default_rng(M)
    N, P = 12, 3
    A, B, C, d = block_system(rng, N, P, M)
    u = oracle.btsv(A, B, C, d, N, P, M, layout=0, transpose=transpose).reshape(N, P, M)
    for p in range(P):
        ud = dense_block(A, B, C, d, p, transpose)
        assert np.abs(u[:, p] - ud).max() < 1e-13 * max(1, np.abs(ud).max())
    # the system-major layout gives the same answer
    to_sm = lambda X: np.ascontiguousarray(np.swapaxes(X, 0, 1))
    u2 = oracle.btsv(to_sm(A), to_sm(B), to_sm(C), to_sm(d), N, P, M, layout=1,
                     transpose=transpose).reshape(P, N, M)
    assert np.array_equal(np.swapaxes(u2, 0, 1), u)


@needs_ref
@pytest.mark.parametrize("M", [2, 3, 4, 8])
def test_block_oracle_pinned_to_reference_gold(M):
    """The reference gold (blktrid_cpu.cpp:388-495) is exact wherever its
    defective matrix product (:301-326, reads M2[i][j] for M2[k][j]) equals
    the true product, i.e. whenever the left operand is diagonal or either
    operand is zero: a single block row (N=1); lower block-bidiagonal systems
    (C=0, dense A and B: every product has a zero operand); upper
    block-bidiagonal systems with diagonal B (A=0: every left operand is
    diagonal or zero).  Our restatement must agree with it there, and
    disagree with it (being right) on general systems."""
    rng = np.random.default_rng(20 + M)
    to_sm = lambda X: np.ascontiguousarray(np.swapaxes(X, 0, 1))
    P, N = 4, 16
    eye = np.eye(M, dtype=bool)

    def both(A, B, C, d, N):
        args = (to_sm(A), to_sm(B), to_sm(C), to_sm(d), N, P, M)
        return oracle.ref_btsv_system_major(*args), oracle.btsv(*args, layout=1)

    ref, ours = both(*block_system(rng, 1, P, M), 1)                 # (1) N = 1
    assert np.abs(ref - ours).max() < 1e-14
    A, B, C, d = block_system(rng, N, P, M)                          # (2) C = 0
    ref, ours = both(A, B, np.zeros_like(C), d, N)
    assert np.abs(ref - ours).max() < 1e-13
    A, B, C, d = block_system(rng, N, P, M)                          # (3) A = 0, diag B
    ref, ours = both(np.zeros_like(A), np.where(eye, B, 0.0), C, d, N)
    assert np.abs(ref - ours).max() < 1e-13
    A, B, C, d = block_system(rng, N, P, M)                          # general blocks
    ref, ours = both(A, B, C, d, N)
    dense = np.stack([dense_block(A, B, C, d, p) for p in range(P)])
    assert np.abs(ours.reshape(P, N, M) - dense).max() < 1e-13
    assert np.abs(ref.reshape(P, N, M) - dense).max() > 1e-6


@needs_ref
def test_adi_oracle_matches_reference_gold():
    """apps/adi/src/adi_orig.c (reference coefficients and initial state)."""
    nx, ny, nz, it = 20, 14, 11, 3
    with tempfile.TemporaryDirectory() as tmp:
        gold = oracle.run_adi_orig(nx, ny, nz, it, tmp)
    u0 = np.zeros((nz, ny, nx))
    u0[[0, -1], :, :] = 1
    u0[:, [0, -1], :] = 1
    u0[:, :, [0, -1]] = 1
    lam = 1.0
    ours = oracle.adi(u0.ravel(), nx, ny, nz, it, lam, -0.5 * lam, 1 + lam, -0.5 * lam)
    assert np.abs(ours - gold).max() <= 1e-13 * np.abs(gold).max()
