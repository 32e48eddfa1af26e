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
(`span`: only the chunks holding rows take part); and the two facts the
adjoint and forward+adjoint kernels build on: the continuant recurrence
(chunk_reduce_cont) gives the Thomas pivots, and the transposed system reuses
them (chunk_reduce_given).  The long-system level on top (warp_block_basis,
block_rows: blocks of 32 chunks reduced to two rows each, the block system
solved at the next level) is checked the same way, and so is the
one-CTA-per-system form whose block system is solved by the odd-even step
plus PCR over the warps.
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


def interior_pivots(al, be, ga):
    """Reciprocal Thomas pivots 1/p_j (j = 1..M-2) of each chunk's interior,
    p_1 = b_1, p_j = b_j - a_j c_{j-1} / p_{j-1} (chunk_reduce_pivots)."""
    M = al.shape[1]
    rp = np.zeros_like(al)
    p = be[:, 1].copy()
    rp[:, 1] = 1.0 / p
    for j in range(2, M - 1):
        p = be[:, j] - al[:, j] * ga[:, j - 1] / p
        rp[:, j] = 1.0 / p
    return rp


def pow2_inv_exponent(x):
    """2^-e for x = m 2^e with m in [1, 2) (x normal, nonzero), else 1."""
    m, k = np.frexp(x)
    return np.where((x != 0) & np.isfinite(x), np.ldexp(1.0, 1 - k), 1.0)


def continuant_pivots(al, be, ga):
    """The same pivots from the continuant recurrence q_j = b_j q_{j-1} -
    (a_j c_{j-1}) q_{j-2}, 1/p_j = q_{j-1} / q_j, the pair rescaled by a power
    of two every 4 rows (chunk_reduce_cont)."""
    M = al.shape[1]
    rp = np.zeros_like(al)
    qm2, qm1 = np.ones(al.shape[0]), be[:, 1].copy()
    rp[:, 1] = 1.0 / be[:, 1]
    for j in range(2, M - 1):
        q = be[:, j] * qm1 - (al[:, j] * ga[:, j - 1]) * qm2
        rp[:, j] = qm1 / q
        qm2, qm1 = qm1, q
        if j % 4 == 0:
            sc = pow2_inv_exponent(q)
            qm1, qm2 = qm1 * sc, qm2 * sc
    return rp


def chunk_reduce_given(al, be, ga, de, rp):
    """chunk_reduce with the interior's reciprocal pivots given."""
    M = al.shape[1]
    ga[:, 1] *= rp[:, 1]
    de[:, 1] *= rp[:, 1]
    al[:, 1] *= rp[:, 1]
    for j in range(2, M - 1):
        r = rp[:, j]
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
    out[:v.size - s] = v[s:]
    return out


def up(v, s):
    """__shfl_up_sync by s (lanes below s read lane 0's value; every use is
    masked there)."""
    out = np.empty_like(v)
    out[s:] = v[:v.size - s]
    out[:s] = v[:s]
    return out


def interface_solve(F, L, span=W):
    """warp_interface_solve over len(F[0]) lanes (32 for a warp; the number
    of warps for the one-CTA kernel's block system)."""
    fa, fb, fc, fd = F
    la, lb, lc, ld = L
    nl = fa.size
    lane = np.arange(nl)
    ifb = 1.0 / fb
    nfa, nfi, nfc, nfd = down(fa, 1, 0.0), down(ifb, 1, 1.0), down(fc, 1, 0.0), down(fd, 1, 0.0)
    p, q = la * ifb, lc * nfi
    ra, rb, rc, rd = -p * fa, lb - p * fc - q * nfa, -q * nfc, ld - p * fd - q * nfd
    s = 1
    while s < nl and s < span:
        ib = 1.0 / rb
        sa, sc, sd = ra * ib, rc * ib, rd * ib
        k1 = np.where(lane >= s, ra, 0.0)
        k2 = np.where(lane + s < nl, rc, 0.0)
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


def chunks(a, b, c, d, M):
    n, rows = a.size, W * M
    t = np.result_type(a, b, c, d)
    al, be, ga, de = (np.zeros(rows, t), np.ones(rows, t), np.zeros(rows, t), np.zeros(rows, t))
    al[1:n], be[:n], ga[:n - 1], de[:n] = a[1:], b, c[:-1], d  # a_0, c_{n-1} never read
    return [v.reshape(W, M) for v in (al, be, ga, de)]


def partition_solve(a, b, c, d, M, span=W, rp=None):
    n = a.size
    al, be, ga, de = chunks(a, b, c, d, M)
    F, L = chunk_reduce(al, be, ga, de) if rp is None else chunk_reduce_given(al, be, ga, de, rp)
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


@pytest.mark.parametrize("M", [4, 8, 16])
def test_continuant_pivots_and_transpose_reuse(M):
    """The continuant pivots equal the Thomas pivots, and the transposed
    system (sub-diagonal c_{i-1}, super-diagonal a_{i+1}) solved with the
    forward chunks' pivots matches the oracle's solve of the transpose: the
    pivots depend on a_j c_{j-1} only."""
    n = W * M
    rng = np.random.default_rng(M)
    a, b, c, d = rand_coeffs(rng, n)
    al, be, ga, _ = chunks(a, b, c, d, M)
    rp = interior_pivots(al, be, ga)
    rc = continuant_pivots(al, be, ga)
    assert np.abs(rc[:, 1:M - 1] - rp[:, 1:M - 1]).max() / np.abs(rp).max() < 1e-14
    x = partition_solve(a, b, c, d, M, rp=rc)
    expect = oracle.mtsv(a, b, c, d, dims=[n], solvedim=0)
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13
    at, ct = np.zeros(n), np.zeros(n)
    at[1:], ct[:-1] = c[:-1], a[1:]
    w = rng.standard_normal(n)
    g = partition_solve(at, b, ct, w, M, rp=rc)
    gexp = oracle.mtsv(at, b, ct, w, dims=[n], solvedim=0)
    assert np.abs(g - gexp).max() / np.abs(gexp).max() < 1e-13


def interface_solve_n(F, L, dF, dL):
    """warp_interface_solve_n: the interface elimination with several
    right-hand sides (dF, dL: [NR, W])."""
    fa, fb, fc, _ = F
    la, lb, lc, _ = L
    lane = np.arange(W)
    ifb = 1.0 / fb
    nfa, nfi, nfc = down(fa, 1, 0.0), down(ifb, 1, 1.0), down(fc, 1, 0.0)
    nfd = np.stack([down(v, 1, 0.0) for v in dF])
    p, q = la * ifb, lc * nfi
    ra, rb, rc = -p * fa, lb - p * fc - q * nfa, -q * nfc
    rd = dL - p * dF - q * nfd
    s = 1
    while s < W:
        ib = 1.0 / rb
        sa, sc = ra * ib, rc * ib
        k1 = np.where(lane >= s, ra, 0.0)
        k2 = np.where(lane + s < W, rc, 0.0)
        ua, uc, da, dc = up(sa, s), up(sc, s), down(sa, s, 0.0), down(sc, s, 0.0)
        sd = rd * ib
        rd = rd - k1 * np.stack([up(v, s) for v in sd]) - k2 * np.stack([down(v, s, 0.0) for v in sd])
        ra, rc = -k1 * ua, -k2 * dc
        rb = rb - k1 * uc - k2 * da
        s <<= 1
    xL = rd / rb
    lprev = np.stack([up(v, 1) for v in xL])
    xF = (dF - np.where(lane > 0, fa * lprev, 0.0) - fc * xL) * ifb
    return xF, xL


def block_basis(F, L):
    """warp_block_basis: lane 0's F row and lane 31's L row replaced by
    identity rows; right-hand sides (d, e_{F^B}, e_{L^B}) give every interface
    unknown as P + F^B UF + L^B UL ([3, W] for the F and L unknowns)."""
    F3 = [v.copy() for v in F]
    L3 = [v.copy() for v in L]
    dF = np.stack([F[3], np.zeros(W), np.zeros(W)])
    dL = np.stack([L[3], np.zeros(W), np.zeros(W)])
    F3[0][0], F3[1][0], F3[2][0] = 0.0, 1.0, 0.0
    dF[:, 0] = (0.0, 1.0, 0.0)
    L3[0][-1], L3[1][-1], L3[2][-1] = 0.0, 1.0, 0.0
    dL[:, -1] = (0.0, 0.0, 1.0)
    return interface_solve_n(F3, L3, dF, dL)


def block_rows(F, L, bF, bL):
    """The block's two reduced rows (block_rows) from lane 0's F row, lane
    31's L row and the basis."""
    fa, fb, fc, fd = (v[0] for v in F)
    la, lb, lc, ld = (v[-1] for v in L)
    l0P, l0F, l0L = bL[:, 0]
    f31P, f31F, f31L = bF[:, -1]
    FB = (fa, fb + fc * l0F, fc * l0L, fd - fc * l0P)
    LB = (la * f31F, lb + la * f31L, lc, ld - la * f31P)
    return FB, LB


def blocked_solve(a, b, c, d, M):
    """Blocks of 32*M rows: chunk reduction, block basis and block rows per
    block, the block system (2 rows per block) by the oracle's Thomas, then
    the interface unknowns from the basis and the chunk interiors."""
    n = a.size
    B = -(-n // (W * M))
    rows = B * W * M
    al, be, ga, de = np.zeros(rows), np.ones(rows), np.zeros(rows), np.zeros(rows)
    al[1:n], be[:n], ga[:n - 1], de[:n] = a[1:], b, c[:-1], d
    blocks = []
    ra, rb, rc, rd = (np.zeros(2 * B) for _ in range(4))
    for k in range(B):
        sl = slice(k * W * M, (k + 1) * W * M)
        ch = [v[sl].reshape(W, M).copy() for v in (al, be, ga, de)]
        F, L = chunk_reduce(*ch)
        bF, bL = block_basis(F, L)
        FB, LB = block_rows(F, L, bF, bL)
        ra[2 * k], rb[2 * k], rc[2 * k], rd[2 * k] = FB
        ra[2 * k + 1], rb[2 * k + 1], rc[2 * k + 1], rd[2 * k + 1] = LB
        blocks.append((ch, bF, bL))
    xb = oracle.mtsv(ra, rb, rc, rd, dims=[2 * B], solvedim=0)
    out = []
    for k, (ch, bF, bL) in enumerate(blocks):
        fB, lB = xb[2 * k], xb[2 * k + 1]
        xF = bF[0] + fB * bF[1] + lB * bF[2]
        xL = bL[0] + fB * bL[1] + lB * bL[2]
        out.append(chunk_backsub(ch[0], ch[2], ch[3], xF, xL).ravel())
    return np.concatenate(out)[:n]


@pytest.mark.parametrize("M", [4, 8])
@pytest.mark.parametrize("nblocks,ragged", [(1, 0), (3, 0), (5, 77), (9, 255)])
def test_blocked_partition_matches_oracle(M, nblocks, ragged):
    """The long-system method (warp_block_basis + block_rows, the block
    system solved at the next level): whole and ragged last blocks."""
    n = nblocks * W * M - ragged
    rng = np.random.default_rng(n + M)
    a, b, c, d = rand_coeffs(rng, n)
    expect = oracle.mtsv(a, b, c, d, dims=[n], solvedim=0)
    x = blocked_solve(a, b, c, d, M)
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13


def cta_solve(a, b, c, d, M, warps):
    """The one-CTA-per-system form (513..4096 rows): a block of 32 chunks per
    warp with its basis and two rows, the 2*warps-row block system solved by
    the same odd-even step plus PCR over the warps (lanes = warps), then every
    warp's interface unknowns and chunk interiors."""
    n = a.size
    rows = warps * W * M
    assert n <= rows
    al, be, ga, de = np.zeros(rows), np.ones(rows), np.zeros(rows), np.zeros(rows)
    al[1:n], be[:n], ga[:n - 1], de[:n] = a[1:], b, c[:-1], d
    blocks, FBs, LBs = [], [], []
    for k in range(warps):
        sl = slice(k * W * M, (k + 1) * W * M)
        ch = [v[sl].reshape(W, M).copy() for v in (al, be, ga, de)]
        F, L = chunk_reduce(*ch)
        bF, bL = block_basis(F, L)
        FB, LB = block_rows(F, L, bF, bL)
        FBs.append(FB)
        LBs.append(LB)
        blocks.append((ch, bF, bL))
    FBw = tuple(np.array([r[i] for r in FBs]) for i in range(4))
    LBw = tuple(np.array([r[i] for r in LBs]) for i in range(4))
    fB, lB = interface_solve(FBw, LBw)
    out = []
    for k, (ch, bF, bL) in enumerate(blocks):
        xF = bF[0] + fB[k] * bF[1] + lB[k] * bF[2]
        xL = bL[0] + fB[k] * bL[1] + lB[k] * bL[2]
        out.append(chunk_backsub(ch[0], ch[2], ch[3], xF, xL).ravel())
    return np.concatenate(out)[:n]


@pytest.mark.parametrize("warps", [2, 4, 8])
@pytest.mark.parametrize("short", [0, 100])
def test_one_cta_block_system_by_pcr_over_warps(warps, short):
    n = warps * W * 16 - short
    rng = np.random.default_rng(warps * 7 + short)
    a, b, c, d = rand_coeffs(rng, n)
    expect = oracle.mtsv(a, b, c, d, dims=[n], solvedim=0)
    x = cta_solve(a, b, c, d, 16, warps)
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13


@pytest.mark.parametrize("M", [4, 8])
def test_partitioned_thomas_in_complex_arithmetic(M):
    """The same equations in complex arithmetic (the complex kernels
    instantiate partition.cuh for a complex type) against the complex
    oracle."""
    from helpers import rand_complex_coeffs
    n = W * M - 5
    rng = np.random.default_rng(M + 100)
    a, b, c, d = rand_complex_coeffs(rng, n)
    expect = oracle.mtsv(a, b, c, d, dims=[n], solvedim=0)
    x = partition_solve(a, b, c, d, M)
    assert np.abs(x - expect).max() / np.abs(expect).max() < 1e-13
