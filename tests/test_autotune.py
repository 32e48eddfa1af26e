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
