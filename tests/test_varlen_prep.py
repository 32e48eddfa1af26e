"""The variable-length batch's preparation restated in numpy (CPU): the
length classes and the work tables the three preparation launches build
(varlen_prep_count / _scan / _fill in tridsolver_b200/csrc/kern_varlen.cu).

Systems of at most 256 rows go to the short queue, in system order (a prefix
scan); 257 .. 4096 rows to the one-CTA bucket ceil(len/512) - 1; 4097 ..
8192 rows to the long list; empty systems nowhere; malformed offsets and
longer systems nowhere, with their error bits.  These tests pin the facts
the kernels rely on: every system lands in at most one table, so no table
index can reach nsys whatever the offsets hold (decreasing, out of range,
or 0, T, 0, T, ... overlapping), and every solvable system lands in exactly
one.
"""

import numpy as np
import pytest

SHORT = 256
MID = 512 * 8       # one-CTA buckets: 8 of them, 512 rows per warp
LONGEST = 256 * 32  # longest solvable system
ERR_BAD, ERR_TOO_LONG = 4, 8
N_LISTS = 9         # the 8 buckets, then the long list


def classify(offsets, total):
    """Per system: ('short', None), ('list', index), ('empty', None),
    ('bad', None) or ('long+', None) -- vl_class."""
    lo, hi = offsets[:-1], offsets[1:]
    out = []
    for a, b in zip(lo, hi):
        if b < a or a < 0 or b > total:
            out.append(("bad", None))
        elif b == a:
            out.append(("empty", None))
        elif b - a <= SHORT:
            out.append(("short", None))
        elif b - a <= MID:
            out.append(("list", int((b - a + 511) // 512) - 1))
        elif b - a <= LONGEST:
            out.append(("list", N_LISTS - 1))
        else:
            out.append(("long+", None))
    return out


def prepare(offsets, total):
    """The tables as the preparation leaves them: (short queue, lists, error
    bits).  List order is the order of arrival (atomic appends), so the lists
    are compared as sets."""
    offsets = np.asarray(offsets, dtype=np.int64)
    nsys = offsets.size - 1
    cls = classify(offsets, total)
    queue = [s for s, (k, _) in enumerate(cls) if k == "short"]  # the prefix scan keeps order
    lists = [[] for _ in range(N_LISTS)]
    err = 0
    for s, (k, li) in enumerate(cls):
        if k == "list":
            lists[li].append(s)
        elif k == "bad":
            err |= ERR_BAD
        elif k == "long+":
            err |= ERR_TOO_LONG
    assert len(queue) <= nsys and all(len(x) <= nsys for x in lists)
    return queue, lists, err


def test_monotone_offsets_every_system_once():
    rng = np.random.default_rng(0)
    for trial in range(200):
        nsys = int(rng.integers(1, 400))
        lens = np.floor(np.exp(rng.uniform(0, np.log(8192), nsys))).astype(np.int64)
        lens[rng.random(nsys) < 0.1] = 0
        off = np.concatenate([[0], np.cumsum(lens)])
        total = int(off[-1]) + int(rng.integers(0, 1000))
        queue, lists, err = prepare(off, total)
        assert err == 0
        seen = queue + [s for x in lists for s in x]
        assert sorted(seen) == [s for s in range(nsys) if lens[s] > 0]
        assert queue == sorted(queue)
        for li, x in enumerate(lists[:-1]):
            assert all(SHORT < lens[s] <= MID and (lens[s] + 511) // 512 == li + 1 for s in x)
        assert all(MID < lens[s] <= LONGEST for s in lists[-1])


def test_alternating_offsets_stay_within_nsys():
    # 0, T, 0, T, ...: systems 0, 2, 4, ... valid and T rows long (a block
    # layout would have asked for far more entries than the tables hold), the
    # others decreasing
    for T in (100, 3000, 8192):
        nsys = 301
        off = np.array([0 if k % 2 == 0 else T for k in range(nsys + 1)], dtype=np.int64)
        queue, lists, err = prepare(off, T)
        assert err == ERR_BAD
        valid = list(range(0, nsys, 2))
        assert sorted(queue + [s for x in lists for s in x]) == valid


def test_too_long_systems_are_flagged_not_listed():
    off = np.array([0, 100, 100 + 8193, 100 + 8193 + 8192], dtype=np.int64)
    queue, lists, err = prepare(off, int(off[-1]))
    assert err == ERR_TOO_LONG
    assert queue == [0] and lists[-1] == [2] and all(not x for x in lists[:-1])


@pytest.mark.parametrize("seed", range(5))
def test_random_malformed_offsets_stay_in_bounds(seed):
    rng = np.random.default_rng(100 + seed)
    nsys = 500
    total = int(rng.integers(1000, 200000))
    off = rng.integers(0, total + 1, nsys + 1)
    off[rng.random(nsys + 1) < 0.02] = total + 5
    off[rng.random(nsys + 1) < 0.02] = -3
    queue, lists, err = prepare(off, total)
    assert err & ERR_BAD
    # every entry names a valid system of its class, each at most once
    seen = queue + [s for x in lists for s in x]
    assert len(seen) == len(set(seen))
    for s in seen:
        assert 0 <= off[s] <= off[s + 1] <= total
