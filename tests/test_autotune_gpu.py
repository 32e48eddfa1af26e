"""The autotuner on the GPU: a sweep of two length buckets of one stride
class and of the variable-length buckets writes a table that, loaded
through tridLoadTuningTable, steers the dispatcher (tridQueryMethod reports
the winners) and the steered solves still match the oracle."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from tridsolver_b200 import autotune  # noqa: E402
from tridsolver_b200.varlen import solve_varlen  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import dev, host, rand_coeffs, rel_err  # noqa: E402


def query(L, dtype_bytes, axis, n):
    m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.tridQueryMethod(dtype_bytes, axis, n, ctypes.byref(m), ctypes.byref(ch),
                             ctypes.byref(spc)) == 0
    return m.value, ch.value, spc.value


def test_sweep_writes_a_table_that_steers_dispatch(tmp_path):
    L = tb.lib()
    table, report = autotune.tune(dtypes=("f64",), lengths=(64, 128), elems=1 << 21,
                                  verbose=False, classes=(1,))
    assert [(t[0], t[1], t[2]) for t in table] == [("f64", 1, 64), ("f64", 1, 128)]
    # every candidate plus the built-in choice of each bucket
    assert len(report) == sum(len(autotune.candidates(1, n)) + 1 for n in (64, 128))
    path = tmp_path / "tuning.txt"
    autotune.write_table(table, str(path))
    assert L.tridLoadTuningTable(str(path).encode()) == 0
    try:
        for _, axis, n, (m, ch, spc) in table:
            got = query(L, 8, axis, n)
            assert got[0] == m, (n, got)
            if m >= 2:  # the dispatcher widens a chunk too small for n
                assert got[2] == (spc if spc else 8) and got[1] >= ch, (n, got)
        # solves through the steered dispatch match the oracle
        rng = np.random.default_rng(4)
        for n in (64, 128):
            dims = [40, n, 5]
            a, b, c, d = rand_coeffs(rng, int(np.prod(dims)))
            expect = oracle.mtsv(a, b, c, d, dims=dims, solvedim=1)
            td = dev(d)
            assert tb.tridDmtsvStridedBatch(dev(a), dev(b), dev(c), td, None, 3, 1, dims,
                                            dims) == 0
            assert rel_err(host(td), expect) <= 1e-12
    finally:
        assert L.tridLoadTuningTable(None) == 0


def test_varlen_bucket_sweep_steers_the_batch(tmp_path):
    L = tb.lib()
    entries, report = autotune.tune_varlen("f64", nsys=20_000, reps=3, verbose=False)
    assert len(report) == len(autotune.VARLEN_BUCKETS)
    path = tmp_path / "vl.txt"
    autotune.write_table(entries, str(path))
    assert L.tridLoadTuningTable(str(path).encode()) == 0
    try:
        best = min(report, key=lambda r: r["ms"])
        for n in (8, 40, 64, 100, 128, 200):
            want = 2 if n <= best["m2max"] else (4 if n <= best["m4max"] else 8)
            assert query(L, 8, 4, n)[1] == want, (n, best)
        rng = np.random.default_rng(6)
        lens = rng.integers(1, 257, 3000)
        off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        a, b, c, d = rand_coeffs(rng, int(off[-1]))
        expect = oracle.varlen(a, b, c, d, off)
        t = [dev(x) for x in (a, b, c, d)]
        solve_varlen(*t, dev(off))
        assert rel_err(host(t[3]), expect) <= 1e-12
    finally:
        assert L.tridLoadTuningTable(None) == 0
