"""Block-tridiagonal batched solve and adjoint (GPU, through the C ABI).

Compared with the corrected block-Thomas oracle (oracle_btsv_f64, which the
CPU tests pin to dense LU and to the reference block gold where that gold is
exact) on the benchmark's block distribution: off-diagonal entries
U(-1,1)/M, diagonal blocks U(-1,1)/M + (2+U(0,1)) I, RHS N(0,1).
Bars: FP64 1e-12 relative max-norm, FP32 1e-5.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from tridsolver_b200 import block  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import rel_err  # noqa: E402


def block_system(rng, N, P, M):
    A = rng.uniform(-1, 1, (N, P, M, M)) / M
    B = rng.uniform(-1, 1, (N, P, M, M)) / M + (2 + rng.uniform(0, 1, (N, P, 1, 1))) * np.eye(M)
    C = rng.uniform(-1, 1, (N, P, M, M)) / M
    d = rng.standard_normal((N, P, M))
    return A, B, C, d


def cuda(x, dtype=np.float64):
    return torch.from_numpy(np.ascontiguousarray(x.astype(dtype))).cuda()


@pytest.mark.parametrize("M", [1, 2, 3, 4, 5, 7, 8, 10])
@pytest.mark.parametrize("N,P", [(1, 33), (2, 5), (17, 100), (256, 40)])
def test_block_solve_fp64(M, N, P):
    rng = np.random.default_rng(M * 1000 + N + P)
    A, B, C, d = block_system(rng, N, P, M)
    expect = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    x = block.btsv(cuda(A), cuda(B), cuda(C), cuda(d))
    assert rel_err(x.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("M", [2, 4, 8])
def test_block_solve_fp32(M):
    rng = np.random.default_rng(M)
    N, P = 64, 70
    A, B, C, d = block_system(rng, N, P, M)
    expect = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    x = block.btsv(*(cuda(v, np.float32) for v in (A, B, C, d)))
    assert rel_err(x.cpu().numpy(), expect) <= 1e-5


def test_block_caller_scratch_and_unused_blocks():
    """Caller-provided Cstar/dstar (the reference API's scratch); A_0 and
    C_{N-1} are never read."""
    rng = np.random.default_rng(3)
    N, P, M = 9, 11, 4
    A, B, C, d = block_system(rng, N, P, M)
    expect = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    A2, C2 = A.copy(), C.copy()
    A2[0] = np.nan
    C2[N - 1] = np.inf
    Cs = torch.empty(N * P * M * M, dtype=torch.float64, device="cuda")
    ds = torch.empty(N * P * M, dtype=torch.float64, device="cuda")
    x = block.btsv(cuda(A2), cuda(B), cuda(C2), cuda(d), Cstar=Cs, dstar=ds)
    assert rel_err(x.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("M", [2, 3, 4])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_block_register_unused_blocks_and_misaligned(dtype, tol, M):
    """M = 2..4 (one thread per system; for M = 2, 4 only when every array is
    16-byte aligned): A_0 and C_{N-1} are never read; arrays one element off
    a 16-byte boundary take the M-lanes kernel (M = 2, 4) and give the same
    answer."""
    rng = np.random.default_rng(22 + M)
    N, P = 37, 300
    A, B, C, d = block_system(rng, N, P, M)
    expect = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    A2, C2 = A.copy(), C.copy()
    A2[0] = np.nan
    C2[N - 1] = np.inf
    x = block.btsv(*(cuda(v, dtype) for v in (A2, B, C2, d)))
    assert rel_err(x.cpu().numpy(), expect) <= tol

    def off(v):  # the same values one element past a 16-byte boundary
        flat = np.concatenate([[0.0], v.ravel()]).astype(dtype)
        return torch.from_numpy(flat).cuda()[1:].view(v.shape)

    x2 = block.btsv(off(A2), off(B), off(C2), off(d), x=off(np.zeros_like(d)))
    assert rel_err(x2.cpu().numpy(), expect) <= tol


def test_reference_cxx_entry_point():
    """dbtsv_gpu(A, B, C, d, Cstar, dstar, u, N, P, blkdim) with C++ linkage."""
    rng = np.random.default_rng(4)
    N, P, M = 8, 13, 3
    A, B, C, d = block_system(rng, N, P, M)
    expect = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    t = [cuda(v) for v in (A, B, C, d)]
    Cs = torch.empty(N * P * M * M, dtype=torch.float64, device="cuda")
    ds = torch.empty(N * P * M, dtype=torch.float64, device="cuda")
    u = torch.zeros(N, P, M, dtype=torch.float64, device="cuda")
    f = getattr(tb.lib(), "_Z9dbtsv_gpuPdS_S_S_S_S_S_iii")
    f.restype = None
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    f(p(t[0]), p(t[1]), p(t[2]), p(t[3]), p(Cs), p(ds), p(u), N, P, M)
    torch.cuda.synchronize()
    assert rel_err(u.cpu().numpy(), expect) <= 1e-12


@pytest.mark.parametrize("M", [1, 2, 3, 4, 8])
def test_block_adjoint(M):
    rng = np.random.default_rng(50 + M)
    N, P = 12, 9
    A, B, C, d = block_system(rng, N, P, M)
    w = rng.standard_normal((N, P, M))
    u = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    g = oracle.btsv(A, B, C, w, N, P, M, layout=0, transpose=True).reshape(N, P, M)
    exp_dA = -np.einsum("npi,npj->npij", g, np.concatenate([np.zeros((1, P, M)), u[:-1]]))
    exp_dB = -np.einsum("npi,npj->npij", g, u)
    exp_dC = -np.einsum("npi,npj->npij", g, np.concatenate([u[1:], np.zeros((1, P, M))]))
    dA, dB, dC, dd = block.btsv_adjoint(cuda(A), cuda(B), cuda(C), cuda(u), cuda(w))
    assert rel_err(dd.cpu().numpy(), g) <= 1e-12
    assert rel_err(dA.cpu().numpy(), exp_dA) <= 1e-12
    assert rel_err(dB.cpu().numpy(), exp_dB) <= 1e-12
    assert rel_err(dC.cpu().numpy(), exp_dC) <= 1e-12


def test_block_autograd_against_dense():
    rng = np.random.default_rng(8)
    N, P, M = 10, 4, 4
    A, B, C, d = block_system(rng, N, P, M)
    w = torch.randn(N, P, M, dtype=torch.float64, device="cuda")
    leaves = [cuda(v).requires_grad_(True) for v in (A, B, C, d)]
    x = block.block_trid_solve(*leaves)
    (x * w).sum().backward()
    ref = [cuda(v).requires_grad_(True) for v in (A, B, C, d)]
    K = torch.zeros(P, N * M, N * M, dtype=torch.float64, device="cuda")
    for n in range(N):
        sl = slice(n * M, (n + 1) * M)
        K = K.index_put((torch.arange(P)[:, None, None], torch.arange(n * M, (n + 1) * M)[None, :, None],
                         torch.arange(n * M, (n + 1) * M)[None, None, :]), ref[1][n])
        if n > 0:
            K = K.index_put((torch.arange(P)[:, None, None], torch.arange(n * M, (n + 1) * M)[None, :, None],
                             torch.arange((n - 1) * M, n * M)[None, None, :]), ref[0][n])
        if n < N - 1:
            K = K.index_put((torch.arange(P)[:, None, None], torch.arange(n * M, (n + 1) * M)[None, :, None],
                             torch.arange((n + 1) * M, (n + 2) * M)[None, None, :]), ref[2][n])
        del sl
    rhs = ref[3].permute(1, 0, 2).reshape(P, N * M, 1)
    xd = torch.linalg.solve(K, rhs).reshape(P, N, M).permute(1, 0, 2)
    (xd * w).sum().backward()
    assert rel_err(x.detach().cpu().numpy(), xd.detach().cpu().numpy()) <= 1e-12
    for g1, g2 in zip(leaves, ref):
        err = float((g1.grad - g2.grad).abs().max() / g2.grad.abs().max())
        assert err <= 1e-10, err


@pytest.mark.parametrize("M", [2, 3, 4])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
@pytest.mark.parametrize("aligned", [True, False])
def test_block_adjoint_register_kernels(M, dtype, tol, aligned):
    """The one-thread-per-system adjoints (M = 2..4) over more systems than a
    CTA holds, and with every array one element off a 16-byte boundary (the
    M-lanes kernel for M = 2, 4)."""
    rng = np.random.default_rng(70 + M)
    N, P = 29, 333
    A, B, C, d = block_system(rng, N, P, M)
    w = rng.standard_normal((N, P, M))
    u = oracle.btsv(A, B, C, d, N, P, M, layout=0).reshape(N, P, M)
    g = oracle.btsv(A, B, C, w, N, P, M, layout=0, transpose=True).reshape(N, P, M)
    exp_dA = -np.einsum("npi,npj->npij", g, np.concatenate([np.zeros((1, P, M)), u[:-1]]))
    exp_dB = -np.einsum("npi,npj->npij", g, u)
    exp_dC = -np.einsum("npi,npj->npij", g, np.concatenate([u[1:], np.zeros((1, P, M))]))

    def dev(v):
        if aligned:
            return cuda(v, dtype)
        flat = np.concatenate([[0.0], v.ravel()]).astype(dtype)
        return torch.from_numpy(flat).cuda()[1:].view(v.shape)

    A2, C2 = A.copy(), C.copy()
    A2[0] = np.nan
    C2[N - 1] = np.inf
    dA, dB, dC, dd = block.btsv_adjoint(dev(A2), dev(B), dev(C2), dev(u), dev(w))
    assert rel_err(dd.cpu().numpy(), g) <= tol
    assert rel_err(dA[1:].cpu().numpy(), exp_dA[1:]) <= tol
    assert rel_err(dB.cpu().numpy(), exp_dB) <= tol
    assert rel_err(dC[:-1].cpu().numpy(), exp_dC[:-1]) <= tol
