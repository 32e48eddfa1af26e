"""The split solve's arithmetic restated in numpy (CPU): slabs reduced to
their two end unknowns in affine form of the unknowns just outside them, the
gathered slabs merged into the outside unknowns of each rank's slab, and the
slab then solved as an ordinary system with the couplings moved to its
right-hand side -- the steps of tridsolver_b200/csrc/kern_split.cu
(seg_merge, split_reduce_kernel, split_patch_kernel), which restate the
reference's distributed Thomas (scalar/src/cuda/trid_cuda_mpi.cu:473-583).

Checked against the oracle's whole-system Thomas for random cuts of one
batch into 1..6 slabs, including slabs of a single row (the library asks for
two rows per rank; the arithmetic needs one).
"""

import numpy as np
import pytest

from oracle import oracle

from helpers import rand_coeffs


def row_segments(a, b, c, d):
    """One row as a segment: x_i = y + p x_{i-1} + q x_{i+1}, both ends the
    same row.  Arrays [6, ...] of (y0, p0, q0, y1, p1, q1)."""
    y, p, q = d / b, -a / b, -c / b
    return np.stack([y, p, q, y, p, q])


def seg_merge(S, T):
    """S (left) and T (right) adjacent: eliminate S's last and T's first
    unknown (denominator 1 - q1(S) p0(T))."""
    inv = 1.0 / (1.0 - S[5] * T[1])
    vy, vp, vq = (S[3] + S[5] * T[0]) * inv, S[4] * inv, S[5] * T[2] * inv
    uy, up, uq = T[0] + T[1] * vy, T[1] * vp, T[1] * vq + T[2]
    return np.stack([S[0] + S[2] * uy, S[1] + S[2] * up, S[2] * uq,
                     T[3] + T[4] * vy, T[4] * vp, T[4] * vq + T[5]])


def reduce_slab(a, b, c, d):
    """[6, nsys] numbers of one slab (rows along axis 0 of the inputs)."""
    segs = row_segments(a, b, c, d)
    S = segs[:, 0]
    for i in range(1, a.shape[0]):
        S = seg_merge(S, segs[:, i])
    return S


def outside_unknowns(bnd, rank):
    """The unknowns just left and right of `rank`'s slab from every rank's
    six numbers ([nranks, 6, nsys])."""
    nranks, nsys = bnd.shape[0], bnd.shape[2]
    ly = lq = np.zeros(nsys)
    if rank > 0:
        L = bnd[0]
        for k in range(1, rank):
            L = seg_merge(L, bnd[k])
        ly, lq = L[3], L[5]
    ry = rp = np.zeros(nsys)
    if rank < nranks - 1:
        R = bnd[rank + 1]
        for k in range(rank + 2, nranks):
            R = seg_merge(R, bnd[k])
        ry, rp = R[0], R[1]
    S = bnd[rank]
    m00, m01 = 1.0 - S[1] * lq, -S[2] * rp
    m10, m11 = -S[4] * lq, 1.0 - S[5] * rp
    r0, r1 = S[0] + S[1] * ly + S[2] * ry, S[3] + S[4] * ly + S[5] * ry
    det = m00 * m11 - m01 * m10
    f, e = (r0 * m11 - m01 * r1) / det, (m00 * r1 - m10 * r0) / det
    return ly + lq * f, ry + rp * e


@pytest.mark.parametrize("seed", range(6))
def test_split_arithmetic_reproduces_thomas(seed):
    rng = np.random.default_rng(seed)
    n, nsys = 40, 7
    a, b, c, d = rand_coeffs(rng, (n, nsys))  # rows along axis 0, one system per column
    a[0], c[-1] = 0.0, 0.0
    expect = oracle.mtsv(np.ascontiguousarray(a.T), np.ascontiguousarray(b.T),
                         np.ascontiguousarray(c.T), np.ascontiguousarray(d.T),
                         dims=[n, nsys], solvedim=0).reshape(nsys, n).T
    nranks = 1 + seed
    cuts = np.sort(rng.choice(np.arange(1, n), size=nranks - 1, replace=False))
    bounds = np.concatenate([[0], cuts, [n]])
    bnd = np.stack([reduce_slab(*(v[bounds[r]:bounds[r + 1]] for v in (a, b, c, d)))
                    for r in range(nranks)])
    x = np.empty_like(d)
    for r in range(nranks):
        s0, s1 = bounds[r], bounds[r + 1]
        left, right = outside_unknowns(bnd, r)
        dd = d[s0:s1].copy()
        dd[0] -= a[s0] * left
        dd[-1] -= c[s1 - 1] * right
        aa, cc = a[s0:s1].copy(), c[s0:s1].copy()
        m = s1 - s0
        x[s0:s1] = oracle.mtsv(np.ascontiguousarray(aa.T), np.ascontiguousarray(b[s0:s1].T),
                               np.ascontiguousarray(cc.T), np.ascontiguousarray(dd.T),
                               dims=[m, nsys], solvedim=0).reshape(nsys, m).T
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13
