"""C-ABI boundary checks that need no GPU.

* both shared libraries load and export every function include/*.h declares;
* argument validation happens on the host, before any CUDA call, and returns
  TRID_STATUS_INVALID_VALUE instead of exiting the process as the reference
  does (scalar/src/cuda/trid_cuda.cu:209-219).
"""

import ctypes
import os
import re
import subprocess

import pytest

import tridsolver_b200 as tb
from tridsolver_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

INVALID = 3


def declared_c_functions(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"TRID_EXTERN_C[^;(]*?\b(\w+)\s*\(", text)))


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


@pytest.mark.parametrize("header,lib", [
    ("trid_b200.h", _lib.LIB_MAIN),
    ("trid_b200_cudacompat.h", _lib.LIB_COMPAT),
])
def test_library_exports_every_declared_symbol(header, lib):
    names = declared_c_functions(header)
    assert names, header
    syms = exported(lib)
    missing = [n for n in names if n not in syms]
    assert not missing, missing


def test_reference_block_entry_points_have_cxx_linkage():
    """dbtsv_gpu/sbtsv_gpu keep the reference's C++ signatures
    (block/include/blktrid_gpu.h:38-40)."""
    for lib in (_lib.LIB_MAIN, _lib.LIB_COMPAT):
        syms = exported(lib)
        assert "_Z9dbtsv_gpuPdS_S_S_S_S_S_iii" in syms
        assert "_Z9sbtsv_gpuPfS_S_S_S_S_S_iii" in syms


def test_block_invalid_arguments_rejected():
    import tridsolver_b200.block  # noqa: F401  (registers the signatures)
    p, _keep = _fake()
    L = tb.lib()
    assert L.tridDbtsvBatch(p, p, p, p, p, 4, 2, 11, None, None) == INVALID   # M > 10
    assert L.tridDbtsvBatch(p, p, p, p, p, 0, 2, 2, None, None) == INVALID    # N < 1
    assert L.tridDbtsvBatch(None, p, p, p, p, 4, 2, 2, None, None) == INVALID


def test_extension_headers_exported_by_main_library():
    syms = exported(_lib.LIB_MAIN)
    for header in sorted(os.listdir(INCLUDE)):
        if header in ("trid_b200_cudacompat.h",):
            continue
        for name in declared_c_functions(header):
            assert name in syms, (header, name)


def test_libraries_load_and_bind():
    assert tb.lib() is not None
    assert tb.compat_lib() is not None
    assert tb.lib().tridGetStatusString(3) == b"TRID_STATUS_INVALID_VALUE"


def _fake(n=64):
    # host buffers only stand in for aligned device pointers: every call below
    # is rejected during host-side validation, before any CUDA call.
    buf = (ctypes.c_double * n)()
    return ctypes.addressof(buf), buf


@pytest.mark.parametrize("ndim,solvedim,dims,pads", [
    (0, 0, [4], [4]),            # ndim < 1
    (9, 0, [1] * 9, [1] * 9),    # ndim > 8
    (2, 2, [4, 4], [4, 4]),      # solvedim out of range
    (2, -1, [4, 4], [4, 4]),
    (2, 0, [4, -1], [4, 4]),     # negative extent
    (2, 0, [4, 4], [3, 4]),      # pads < dims
])
def test_invalid_geometry_rejected(ndim, solvedim, dims, pads):
    p, _keep = _fake()
    st = tb.tridDmtsvStridedBatch(p, p, p, p, None, ndim, solvedim, dims, pads)
    assert st == INVALID
    st = tb.tridSmtsvStridedBatchInc(p, p, p, p, p, ndim, solvedim, dims, pads)
    assert st == INVALID


def test_null_and_misaligned_pointers_rejected():
    p, _keep = _fake()
    assert tb.tridDmtsvStridedBatch(p, p, p, None, None, 1, 0, [8], [8]) == INVALID
    assert tb.tridDmtsvStridedBatchInc(p, p, p, p, None, 1, 0, [8], [8]) == INVALID
    assert tb.tridDmtsvStridedBatch(p + 4, p, p, p, None, 1, 0, [8], [8]) == INVALID
    assert tb.tridSmtsvStridedBatch(p + 2, p, p, p, None, 1, 0, [8], [8]) == INVALID


def test_complex_and_mixed_invalid_arguments_rejected():
    p, _keep = _fake()
    q = (p + 15) & ~15  # 16-byte aligned, inside the buffer
    for fn in (tb.tridZmtsvStridedBatch, tb.tridCmtsvStridedBatch, tb.tridSmtsvStridedBatchMixed):
        assert fn(q, q, q, q, None, 0, 0, [4], [4]) == INVALID
        assert fn(q, q, q, q, None, 2, 0, [4, 4], [3, 4]) == INVALID
        assert fn(q, q, q, None, None, 1, 0, [8], [8]) == INVALID
    for fn in (tb.tridZmtsvStridedBatchInc, tb.tridCmtsvStridedBatchInc,
               tb.tridSmtsvStridedBatchMixedInc):
        assert fn(q, q, q, q, None, 1, 0, [8], [8]) == INVALID  # Inc needs u
    # elements aligned to their size: 16 / 8 / 4 bytes
    assert tb.tridZmtsvStridedBatch(q + 8, q, q, q, None, 1, 0, [8], [8]) == INVALID
    assert tb.tridCmtsvStridedBatch(q, q, q, q + 4, None, 1, 0, [8], [8]) == INVALID
    assert tb.tridSmtsvStridedBatchMixed(q, q + 2, q, q, None, 1, 0, [8], [8]) == INVALID


def test_solve_rejects_unsupported_dtypes_on_the_host():
    """solve() checks the element type before any pointer or CUDA call:
    float16 and fp64_arithmetic on non-float32 tensors raise TypeError."""
    torch = pytest.importorskip("torch")
    h = torch.ones(2, 8, dtype=torch.float16)
    with pytest.raises(TypeError):
        tb.solve(h, h, h, h)
    for dt in (torch.float64, torch.complex64, torch.complex128):
        x = torch.ones(2, 8, dtype=dt)
        with pytest.raises(TypeError):
            tb.solve(x, x, x, x, fp64_arithmetic=True)
    x = torch.ones(2, 8, dtype=torch.complex128)  # supported type, host tensor
    with pytest.raises(ValueError):
        tb.solve(x, x, x, x)


def test_component_modules_reject_other_element_types():
    """block, varlen and ADI take float32/float64 only: a complex or float16
    tensor raises TypeError on the host instead of reaching the FP32 entry
    point."""
    torch = pytest.importorskip("torch")
    from tridsolver_b200 import adi, block, varlen
    for dt in (torch.complex128, torch.float16):
        A = torch.ones(3, 2, 2, 2, dtype=dt)
        d = torch.ones(3, 2, 2, dtype=dt)
        with pytest.raises(TypeError):
            block.btsv(A, A, A, d)
        with pytest.raises(TypeError):
            block.btsv_adjoint(A, A, A, d, d)
        v = torch.ones(8, dtype=dt)
        with pytest.raises(TypeError):
            varlen.solve_varlen(v, v, v, v, torch.tensor([0, 8]))
    A64, d32 = torch.ones(3, 2, 2, 2, dtype=torch.float64), torch.ones(3, 2, 2)
    with pytest.raises(TypeError):  # mixed element types
        block.btsv(A64, A64, A64, d32)
    with pytest.raises(TypeError):
        adi.ADI((4, 4, 4), 1.0, dtype=torch.complex128, device="cpu")


def test_complex_and_mixed_empty_problems_are_noops():
    """A zero extent returns SUCCESS before any CUDA call (host buffers stand
    in for device pointers and are left untouched)."""
    p, keep = _fake()
    q = (p + 15) & ~15
    before = list(keep)
    for fn in (tb.tridZmtsvStridedBatch, tb.tridCmtsvStridedBatch, tb.tridSmtsvStridedBatchMixed):
        assert fn(q, q, q, q, None, 2, 0, [0, 10], [0, 10]) == 0
        assert fn(q, q, q, q, None, 2, 1, [10, 0], [10, 0]) == 0
    for fn in (tb.tridZmtsvStridedBatchInc, tb.tridCmtsvStridedBatchInc,
               tb.tridSmtsvStridedBatchMixedInc):
        assert fn(q, q, q, q, q, 3, 2, [4, 4, 0], [4, 4, 0]) == 0
    assert list(keep) == before


def test_bad_opts_rejected_by_padded_and_compat():
    p, _keep = _fake()
    st = tb.tridDmtsvStridedBatchPadded(p, [8], p, [8], p, [8], p, [8], None, [8], 1, 0, [8],
                                        opts=[7], sync=0)
    assert st == INVALID
    L = tb.compat_lib()
    opts = _lib.int_array([9, 0, 0])
    st = L.tridDmtsvStridedBatch(p, p, p, p, None, 1, 0, _lib.int_array([8]),
                                 _lib.int_array([8]), opts, 0)
    assert st == INVALID


def test_method_override_and_query():
    L = tb.lib()
    m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.tridQueryMethod(8, 0, 256, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value) == (2, 8)
    # axis 0 up to 64 rows: plain loads (the sweep's winner over TMA staging)
    for n in (2, 32, 64):
        assert L.tridQueryMethod(8, 0, n, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
        assert m.value == 3, n
    # long systems: blocked partition with 256-row blocks
    assert L.tridQueryMethod(8, 1, 5000, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value) == (2, 8)
    assert L.tridQueryMethod(8, 0, 65536, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value) == (2, 8)
    # FP32 along axis 0: 512-row blocks
    assert L.tridQueryMethod(4, 0, 65536, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value) == (2, 16)
    assert L.tridQueryMethod(4, 1, 65536, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value) == (2, 8)
    # strided axes, every stride class: streamed tiles of one 128-byte line of
    # systems (16 FP64, 32 FP32)
    for cls in (1, 2, 3):
        assert L.tridQueryMethod(8, cls, 256, ctypes.byref(m), ctypes.byref(ch),
                                 ctypes.byref(spc)) == 0
        assert (m.value, ch.value, spc.value) == (2, 8, 16)
        assert L.tridQueryMethod(4, cls, 256, ctypes.byref(m), ctypes.byref(ch),
                                 ctypes.byref(spc)) == 0
        assert (m.value, ch.value, spc.value) == (2, 8, 32)
    assert L.tridQueryMethod(8, 5, 256, ctypes.byref(m), ctypes.byref(ch),
                             ctypes.byref(spc)) == INVALID
    # class 4: the variable-length batch's length buckets (2 / 4 / 8 rows per lane)
    for n, want in ((8, 2), (64, 2), (65, 4), (128, 4), (129, 8), (256, 8), (5000, 8)):
        assert L.tridQueryMethod(8, 4, n, ctypes.byref(m), ctypes.byref(ch),
                                 ctypes.byref(spc)) == 0
        assert (m.value, ch.value) == (2, want), n
    tb.set_method(1)
    assert L.tridQueryMethod(8, 0, 256, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert m.value == 1
    tb.set_method(6)
    assert L.tridQueryMethod(8, 0, 1024, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert m.value == 6
    tb.set_method(0)
    for removed in (4, 5):  # methods that no longer exist
        with pytest.raises(tb.TridError):
            tb.set_method(removed)
    with pytest.raises(tb.TridError):
        tb.set_method(2, chunk=3)
    with pytest.raises(tb.TridError):
        tb.set_method(7)
    with pytest.raises(tb.TridError):
        tb.set_method(2, sys_per_cta=12)
    tb.set_method(2, sys_per_cta=32)
    assert L.tridQueryMethod(4, 2, 256, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, spc.value) == (2, 32)
    tb.set_method(0)


def test_tuning_table_rejects_bad_widths(tmp_path):
    L = tb.lib()
    for line in ("f64 2 256 2 8 12\n", "f64 2 256 2 3 16\n"):
        bad = tmp_path / "bad.txt"
        bad.write_text(line)
        assert L.tridLoadTuningTable(str(bad).encode()) == INVALID
    good = tmp_path / "good.txt"
    good.write_text("f32 2 256 2 8 32\n")
    assert L.tridLoadTuningTable(str(good).encode()) == 0
    m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.tridQueryMethod(4, 2, 200, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc)) == 0
    assert (m.value, ch.value, spc.value) == (2, 8, 32)
    assert L.tridLoadTuningTable(None) == 0


def test_tuning_table_roundtrip(tmp_path):
    L = tb.lib()
    path = tmp_path / "tune.txt"
    path.write_text("# dtype axis nmax method chunk spc\nf64 1 300 2 16 4\nf32 0 100 1 0 0\n")
    assert L.tridLoadTuningTable(str(path).encode()) == 0
    m, ch, spc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.tridQueryMethod(8, 1, 256, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc))
    assert (m.value, ch.value, spc.value) == (2, 16, 4)
    L.tridQueryMethod(4, 0, 64, ctypes.byref(m), ctypes.byref(ch), ctypes.byref(spc))
    assert m.value == 1
    bad = tmp_path / "bad.txt"
    bad.write_text("f16 0 1 1 0 0\n")
    assert L.tridLoadTuningTable(str(bad).encode()) == INVALID
    assert L.tridLoadTuningTable(None) == 0


@pytest.mark.parametrize("header", sorted(h for h in os.listdir(INCLUDE) if h.endswith(".h")))
@pytest.mark.parametrize("lang,compiler,std", [("c", "gcc", "c99"), ("c++", "g++", "c++17")])
def test_headers_compile_for_c_and_cxx_callers(tmp_path, header, lang, compiler, std):
    """Each public header compiles on its own as C99 and C++17 (a caller
    includes trid_b200.h or, for the 11-argument forms, trid_b200_cudacompat.h,
    never both); the complex element types are interleaved (re, im) pairs of
    8 / 16 bytes."""
    import shutil
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    src = tmp_path / ("check.c" if lang == "c" else "check.cpp")
    text = f'#include "{header}"\n'
    if header == "trid_b200.h":
        kw = "_Static_assert" if lang == "c" else "static_assert"
        text += (f"{kw}(sizeof(tridComplexF) == 8, \"complex<float>\");\n"
                 f"{kw}(sizeof(tridComplexD) == 16, \"complex<double>\");\n")
    src.write_text(text)
    r = subprocess.run([compiler, f"-std={std}", "-Wall", "-Werror", "-fsyntax-only", "-I", INCLUDE,
                        "-x", lang, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
