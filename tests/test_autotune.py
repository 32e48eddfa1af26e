"""Autotuner host logic (no GPU): its candidates are exactly what the C ABI
accepts, the streamed full-line widths are offered on strided axes, timing
problems have the stated stride classes, and a written table loads back
through tridLoadTuningTable and steers tridQueryMethod."""

import ctypes

import numpy as np
import pytest

import tridsolver_b200 as tb
from tridsolver_b200 import autotune


@pytest.mark.parametrize("axis", [0, 1, 2, 3])
@pytest.mark.parametrize("n", [2, 32, 100, 256, 300, 512, 1000, 5000])
def test_candidates_accepted_by_abi(axis, n):
    L = tb.lib()
    try:
        for m in autotune.candidates(axis, n):
            assert L.tridSetMethod(*m) == 0, m
    finally:
        L.tridSetMethod(0, 0, 0)


def test_strided_candidates_offer_full_line_tiles():
    c = autotune.candidates(2, 256)
    assert (2, 8, 16) in c and (2, 8, 32) in c  # FP64 / FP32 streamed tiles
    assert (3, 8, 8) in c and (2, 8, 8) in c    # narrow tiles stay in the sweep
    assert all(m[0] != 5 and m[0] != 6 for m in c)


@pytest.mark.parametrize("axis", [0, 1, 2, 3])
def test_problem_dims_stride_class(axis):
    dims, sd = autotune.problem_dims(axis, 256, 1 << 24)
    stride_bytes = int(np.prod(dims[:sd])) * 8
    assert dims[sd] == 256
    if axis == 0:
        assert sd == 0
    elif axis == 1:
        assert stride_bytes <= 64 << 10
    elif axis == 2:
        assert 64 << 10 < stride_bytes <= 1 << 20
    else:
        assert stride_bytes > 1 << 20


def test_written_table_loads_and_steers(tmp_path):
    path = tmp_path / "t.txt"
    autotune.write_table([("f64", 2, 256, (3, 8, 16)), ("f32", 1, 128, (2, 4, 32))], str(path))
    L = tb.lib()
    assert L.tridLoadTuningTable(str(path).encode()) == 0
    try:
        m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        assert L.tridQueryMethod(8, 2, 200, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
        assert (m.value, ch.value, spc.value) == (3, 8, 16)
        assert L.tridQueryMethod(4, 1, 100, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
        assert (m.value, ch.value, spc.value) == (2, 4, 32)
        # outside the table's lengths: the built-in default
        assert L.tridQueryMethod(8, 2, 400, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
        assert (m.value, spc.value) == (2, 16)
    finally:
        assert L.tridLoadTuningTable(None) == 0


def test_varlen_bucket_entries_move_the_cutoffs(tmp_path):
    """Axis-class-4 lines of a tuning table set the variable-length batch's
    length buckets; rows per lane never exceed what 32 lanes hold."""
    path = tmp_path / "vl.txt"
    autotune.write_table([("f64", 4, 32, (2, 2, 0)), ("f64", 4, 200, (2, 4, 0))], str(path))
    L = tb.lib()
    assert L.tridLoadTuningTable(str(path).encode()) == 0
    try:
        m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        got = {}
        for n in (8, 32, 33, 128, 129, 300):
            assert L.tridQueryMethod(8, 4, n, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
            got[n] = ch.value
        # 2 up to 32, 4 up to 128 (the 200 of the table is capped), then 8
        assert got == {8: 2, 32: 2, 33: 4, 128: 4, 129: 8, 300: 8}
        # FP32 keeps the built-in cut-offs (the table names f64 only)
        assert L.tridQueryMethod(4, 4, 33, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
        assert ch.value == 2
    finally:
        assert L.tridLoadTuningTable(None) == 0


def test_varlen_bucket_entries_validated(tmp_path):
    path = tmp_path / "bad.txt"
    path.write_text("f64 4 64 3 2 0\n")  # class 4 takes method 2 only
    assert tb.lib().tridLoadTuningTable(str(path).encode()) == 3
