"""The variable-length batch's preparation restated in numpy (CPU): the
per-system item counts, their prefix sums and the item tables of the reduce
and finish queues (varlen_prep_count / _scan / _fill in
tridsolver_b200/csrc/kern_varlen.cu), including the capacity guard.

The item tables are sized for cap = nsys + total/256 + 1 entries.  These
tests pin the two facts the guard rests on: monotone offsets never need more
than cap items (so no valid input is ever skipped), and offsets that do not
increase monotonically can ask for far more (0, T, 0, T, ...), in which case
every system whose items would end past cap is skipped whole, no table index
reaches cap, and the systems before it keep exactly the items they would
have had without the guard.
"""

import numpy as np
import pytest

BLOCK = 256      # rows per block of a long system
SHORT = 256      # longest system solved as one item
MAX_BLOCKS = 32  # longest solvable system: 32 blocks


def cap_of(nsys, total):
    return nsys + total // BLOCK + 1


def counts(offsets, total, cap):
    """Per-system reduce/finish items (vl_counts), clamped to cap + 1."""
    lo, hi = offsets[:-1], offsets[1:]
    bad = (hi < lo) | (lo < 0) | (hi > total)
    ln = np.where(bad, 0, hi - lo)
    nblk = (ln + BLOCK - 1) // BLOCK
    ni = np.where(ln <= SHORT, 1, nblk)
    nf = np.where((ln > SHORT) & (nblk <= MAX_BLOCKS), nblk, 0)
    return np.minimum(ni, cap + 1), np.minimum(nf, cap + 1), bad


def prepare(offsets, total):
    """Item tables as the three preparation launches leave them.  Returns
    (item_sys, fitem_sys, item_off, fitem_off, skipped, flagged)."""
    offsets = np.asarray(offsets, dtype=np.int64)
    nsys = offsets.size - 1
    cap = cap_of(nsys, total)
    ni, nf, bad = counts(offsets, total, cap)
    ri = np.concatenate([[0], np.cumsum(ni)])
    rf = np.concatenate([[0], np.cumsum(nf)])
    item_sys = np.full(cap, -2, dtype=np.int64)   # -2: never written
    fitem_sys = np.full(cap, -2, dtype=np.int64)
    skipped = np.zeros(nsys, dtype=bool)
    for s in range(nsys):
        fits = ri[s] + ni[s] <= cap and rf[s] + nf[s] <= cap
        skipped[s] = not fits
        tag = s if fits else -1
        for k in range(ri[s], min(ri[s] + ni[s], cap)):
            item_sys[k] = tag
        for k in range(rf[s], min(rf[s] + nf[s], cap)):
            fitem_sys[k] = tag
    flagged = bool(bad.any() or skipped.any())
    return item_sys, fitem_sys, ri, rf, skipped, flagged


def test_monotone_offsets_never_reach_cap():
    rng = np.random.default_rng(0)
    for trial in range(200):
        nsys = int(rng.integers(1, 400))
        # lengths from 0 up to past the longest solvable system
        lens = np.floor(np.exp(rng.uniform(0, np.log(12000), nsys))).astype(np.int64)
        lens[rng.random(nsys) < 0.1] = 0
        off = np.concatenate([[0], np.cumsum(lens)])
        total = int(off[-1]) + int(rng.integers(0, 1000))  # total may exceed the last offset
        cap = cap_of(nsys, total)
        ni, nf, bad = counts(off, total, cap)
        assert not bad.any()
        assert ni.sum() <= cap - 1 and nf.sum() <= ni.sum()
        item_sys, fitem_sys, ri, rf, skipped, flagged = prepare(off, total)
        assert not skipped.any() and not flagged
        # every reduce item names its system, in system order
        assert np.array_equal(item_sys[: ri[-1]], np.repeat(np.arange(nsys), ni))
        assert np.array_equal(fitem_sys[: rf[-1]], np.repeat(np.arange(nsys), nf))


def test_alternating_offsets_are_capped():
    # 0, T, 0, T, ...: systems 0, 2, 4, ... are valid and T rows long, the
    # others decreasing.  Without the guard they would need far more items
    # than cap.
    T, nsys = 8192, 301
    off = np.array([0 if k % 2 == 0 else T for k in range(nsys + 1)], dtype=np.int64)
    cap = cap_of(nsys, T)
    ni, nf, bad = counts(off, T, cap)
    assert ni.sum() > 10 * cap  # what the unguarded tables would have held
    item_sys, fitem_sys, ri, rf, skipped, flagged = prepare(off, T)
    assert flagged
    # no entry at or past cap exists (the tables are cap long) and every entry
    # below the prefix total was written
    assert (item_sys[: min(ri[-1], cap)] != -2).all()
    # systems are skipped from the first one that does not fit onwards
    first = int(np.argmax(skipped))
    assert skipped[first:].all() and not skipped[:first].any()
    # the systems that fit keep their full item range, below cap
    for s in range(first):
        assert ri[s] + ni[s] <= cap
        assert (item_sys[ri[s]: ri[s] + ni[s]] == s).all()
    # the kernel serves min(prefix, cap) items; skipped ones read -1
    served = item_sys[: min(ri[-1], cap)]
    assert set(np.unique(served)) <= set(range(first)) | {-1}


@pytest.mark.parametrize("seed", range(5))
def test_random_malformed_offsets_stay_in_bounds(seed):
    rng = np.random.default_rng(100 + seed)
    nsys = 500
    total = int(rng.integers(1000, 200000))
    off = rng.integers(0, total + 1, nsys + 1)
    # some out of range, some negative
    off[rng.random(nsys + 1) < 0.02] = total + 5
    off[rng.random(nsys + 1) < 0.02] = -3
    item_sys, fitem_sys, ri, rf, skipped, flagged = prepare(off, total)
    cap = cap_of(nsys, total)
    assert item_sys.size == cap and fitem_sys.size == cap
    assert flagged  # random offsets are never monotone here
    # a system served by the kernel fits whole below cap
    for s in np.unique(item_sys[: min(ri[-1], cap)]):
        if s >= 0:
            assert ri[s + 1] <= cap
