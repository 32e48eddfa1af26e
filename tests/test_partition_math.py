"""The partitioned Thomas method of the scalar kernels restated in numpy
(CPU): 32 chunks of M rows per system, each chunk reduced to two interface
rows with its first unknown as a parameter, the 64-row interface system
solved by one odd-even elimination step and parallel cyclic reduction over
the 32 chunks (the warp's lanes), then the chunks' interiors -- the
equations of tridsolver_b200/csrc/partition.cuh (chunk_reduce,
warp_interface_solve, chunk_backsub), lane shuffles written as array shifts.

Checked against the oracle's Thomas (the reference's operation order,
trid_cpu.cpp:360-401) for every chunk size the kernels use, for lengths that
fill the 32 chunks partly (identity rows past n) and for a PCR cut short
(`span`: only the chunks holding rows take part).
"""

import numpy as np
import pytest

from oracle import oracle

from helpers import rand_coeffs

W = 32


def chunk_reduce(al, be, ga, de):
    """[W, M] per system (lane = chunk).  Returns the F and L interface rows
    (each a tuple a, b, c, d of [W] arrays); al/ga/de hold a'_j, c'_j, d'_j."""
    M = al.shape[1]
    if M == 2:
        return tuple(v[:, 0] for v in (al, be, ga, de)), tuple(v[:, 1] for v in (al, be, ga, de))
    r = 1.0 / be[:, 1]
    ga[:, 1] *= r
    de[:, 1] *= r
    al[:, 1] *= r
    for j in range(2, M - 1):
        r = 1.0 / (be[:, j] - al[:, j] * ga[:, j - 1])
        de[:, j] = (de[:, j] - al[:, j] * de[:, j - 1]) * r
        al[:, j] = -(al[:, j] * al[:, j - 1]) * r
        ga[:, j] = ga[:, j] * r
    D, A, C = de[:, M - 2].copy(), al[:, M - 2].copy(), ga[:, M - 2].copy()
    L = (-al[:, M - 1] * A, be[:, M - 1] - al[:, M - 1] * C, ga[:, M - 1].copy(),
         de[:, M - 1] - al[:, M - 1] * D)
    for j in range(M - 3, 0, -1):
        D = de[:, j] - ga[:, j] * D
        A = al[:, j] - ga[:, j] * A
        C = -ga[:, j] * C
    F = (al[:, 0].copy(), be[:, 0] - ga[:, 0] * A, -ga[:, 0] * C, de[:, 0] - ga[:, 0] * D)
    return F, L


def down(v, s, fill):
    """__shfl_down_sync by s (lanes past the end keep `fill`)."""
    out = np.full_like(v, fill)
    out[:W - s] = v[s:]
    return out


def up(v, s):
    """__shfl_up_sync by s (lanes below s read lane 0's value; every use is
    masked there)."""
    out = np.empty_like(v)
    out[s:] = v[:W - s]
    out[:s] = v[:s]
    return out


def interface_solve(F, L, span=W):
    fa, fb, fc, fd = F
    la, lb, lc, ld = L
    lane = np.arange(W)
    ifb = 1.0 / fb
    nfa, nfi, nfc, nfd = down(fa, 1, 0.0), down(ifb, 1, 1.0), down(fc, 1, 0.0), down(fd, 1, 0.0)
    p, q = la * ifb, lc * nfi
    ra, rb, rc, rd = -p * fa, lb - p * fc - q * nfa, -q * nfc, ld - p * fd - q * nfd
    s = 1
    while s < W and s < span:
        ib = 1.0 / rb
        sa, sc, sd = ra * ib, rc * ib, rd * ib
        k1 = np.where(lane >= s, ra, 0.0)
        k2 = np.where(lane + s < W, rc, 0.0)
        ua, uc, ud = up(sa, s), up(sc, s), up(sd, s)
        da, dc, dd = down(sa, s, 0.0), down(sc, s, 0.0), down(sd, s, 0.0)
        ra, rc = -k1 * ua, -k2 * dc
        rb, rd = rb - k1 * uc - k2 * da, rd - k1 * ud - k2 * dd
        s <<= 1
    xL = rd / rb
    lprev = up(xL, 1)
    xF = (fd - np.where(lane > 0, fa * lprev, 0.0) - fc * xL) * ifb
    return xF, xL


def chunk_backsub(al, ga, de, xF, xL):
    M = al.shape[1]
    x = xL.copy()
    for j in range(M - 2, 0, -1):
        x = de[:, j] - al[:, j] * xF - ga[:, j] * x
        de[:, j] = x
    de[:, 0] = xF
    de[:, M - 1] = xL
    return de


def partition_solve(a, b, c, d, M, span=W):
    n = a.size
    rows = W * M
    al, be, ga, de = np.zeros(rows), np.ones(rows), np.zeros(rows), np.zeros(rows)
    al[1:n], be[:n], ga[:n - 1], de[:n] = a[1:], b, c[:-1], d  # a_0, c_{n-1} never read
    al, be, ga, de = (v.reshape(W, M) for v in (al, be, ga, de))
    F, L = chunk_reduce(al, be, ga, de)
    xF, xL = interface_solve(F, L, span)
    return chunk_backsub(al, ga, de, xF, xL).ravel()[:n]


@pytest.mark.parametrize("M", [2, 4, 8, 16])
@pytest.mark.parametrize("fill", [1.0, 0.7, 0.26])
def test_partitioned_thomas_matches_oracle(M, fill):
    n = max(2, int(W * M * fill))
    rng = np.random.default_rng(10 * M + int(fill * 100))
    a, b, c, d = rand_coeffs(rng, n)
    expect = oracle.mtsv(a, b, c, d, dims=[n], solvedim=0)
    x = partition_solve(a, b, c, d, M)
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13
    # PCR stopped after log2(span) steps, span >= the chunks holding rows
    span = 1 << int(np.ceil(np.log2(max(1, -(-n // M)))))
    xs = partition_solve(a, b, c, d, M, span=max(span, 2))
    assert np.abs(xs - expect).max() / np.abs(expect).max() < 1e-13
