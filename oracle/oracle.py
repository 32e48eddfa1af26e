"""ORACLE -- test infrastructure only.

numpy/ctypes front end for the CPU checkers:

* ``liboracle.so``  -- the plain-C restatement in ``trid_oracle.c`` (always built);
* ``_ref/*``        -- the reference's own CPU code compiled unmodified by the
                       ``ref`` target of the Makefile (present wherever it was
                       built; it travels with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import
this module.  The shipped package (tridsolver_b200) never does.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None
_REF_BLK = None

c_i64 = ctypes.c_int64
c_int = ctypes.c_int
c_dbl = ctypes.c_double
vp = ctypes.c_void_p


def build(ref=False):
    """Build liboracle.so (and the reference CPU code when ``ref``)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
    return _LIB


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libtrid_cpu_ref.so"))


def ref_lib():
    global _REF
    if _REF is None:
        # the reference keeps c2/d2[N_MAX] (N_MAX = 65536) of SIMD vectors on
        # every OpenMP thread's stack; libgomp reads this when it loads
        os.environ.setdefault("OMP_STACKSIZE", "64M")
        _REF = ctypes.CDLL(os.path.join(HERE, "_ref", "libtrid_cpu_ref.so"))
    return _REF


def ref_block_lib():
    global _REF_BLK
    if _REF_BLK is None:
        _REF_BLK = ctypes.CDLL(os.path.join(HERE, "_ref", "libblktrid_cpu_ref.so"))
    return _REF_BLK


def _p(x):
    return None if x is None else x.ctypes.data_as(vp)


def _ipad(v):
    return (c_int * len(v))(*[int(t) for t in v])


def _suffix(dtype):
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32",
            np.dtype(np.complex128): "c128", np.dtype(np.complex64): "c64"}[np.dtype(dtype)]


# --------------------------------------------------------------------------- #
# Scalar strided batch (restatement)                                          #
# --------------------------------------------------------------------------- #
def mtsv(a, b, c, d, u=None, ndim=None, solvedim=0, dims=None, pads=None, inc=False,
         array_pads=None):
    """Solve the strided batch on copies; returns the new d (non-Inc) or u (Inc).

    ``pads`` applies to every array unless ``array_pads`` = (ap, bp, cp, dp, up)
    gives each array its own padding (the Padded API).
    """
    dims = [int(v) for v in dims]
    ndim = len(dims) if ndim is None else ndim
    pads = dims if pads is None else [int(v) for v in pads]
    ap = array_pads if array_pads is not None else (pads,) * 5
    d = np.array(d, copy=True)
    u = None if u is None else np.array(u, copy=True)
    f = getattr(lib(), "oracle_mtsv_" + _suffix(d.dtype))
    f.restype = c_int
    st = f(_p(a), _ipad(ap[0]), _p(b), _ipad(ap[1]), _p(c), _ipad(ap[2]), _p(d), _ipad(ap[3]),
           _p(u) if inc else None, _ipad(ap[4]), c_int(ndim), c_int(solvedim), _ipad(dims),
           c_int(1 if inc else 0))
    assert st == 0, st
    return u if inc else d


def trid_scalar(a, b, c, d, u, n, stride, inc=False):
    d = np.array(d, copy=True)
    u = None if u is None else np.array(u, copy=True)
    f = getattr(lib(), "oracle_trid_scalar_" + _suffix(d.dtype))
    f(_p(a), _p(b), _p(c), _p(d), _p(u), c_i64(n), c_i64(stride), c_int(1 if inc else 0))
    return u if inc else d


def varlen(a, b, c, d, offsets, u=None, inc=False):
    d = np.array(d, copy=True)
    u = None if u is None else np.array(u, copy=True)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    f = getattr(lib(), "oracle_varlen_" + _suffix(d.dtype))
    f(_p(a), _p(b), _p(c), _p(d), _p(u), _p(offsets), c_i64(offsets.size - 1),
      c_int(1 if inc else 0))
    return u if inc else d


def adjoint(a, b, c, u, w, n):
    """Adjoint of contiguous systems of length n: returns (g, ga, gb, gc)."""
    a, b, c, u, w = (np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c, u, w))
    nsys = a.size // n
    outs = [np.empty_like(a) for _ in range(4)]
    lib().oracle_adjoint_f64(_p(a), _p(b), _p(c), _p(u), _p(w), *[_p(o) for o in outs],
                             c_i64(n), c_i64(nsys))
    return tuple(outs)


def btsv(A, B, C, d, N, P, M, layout=0, transpose=False):
    """Block tridiagonal solve (layout 0 = interleaved [n][p], 1 = [p][n])."""
    A, B, C, d = (np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, C, d))
    u = np.zeros_like(d)
    st = lib().oracle_btsv_f64(_p(A), _p(B), _p(C), _p(d), _p(u), c_int(N), c_int(P), c_int(M),
                               c_int(layout), c_int(1 if transpose else 0))
    assert st == 0
    return u


def adi(u0, nx, ny, nz, iters, lam, a_int, b_int, c_int_):
    u = np.array(u0, dtype=np.float64, copy=True)
    lib().oracle_adi_f64(_p(u), c_int(nx), c_int(ny), c_int(nz), c_int(iters), c_dbl(lam),
                         c_dbl(a_int), c_dbl(b_int), c_dbl(c_int_))
    return u


# --------------------------------------------------------------------------- #
# The reference CPU library (oracle/_ref)                                      #
# --------------------------------------------------------------------------- #
def _placed(x, aligned):
    """Copy x into a buffer 64-byte aligned (aligned=True) or 8 bytes past a
    64-byte boundary.  The reference dispatcher sends solvedim 0 to its AVX
    transpose path only when every pointer is 64-byte aligned
    (trid_cpu.cpp:418), and that path is wrong; its solvedim 1/2 paths need
    32-byte aligned vectors (trid_cpu.cpp:304-355)."""
    x = np.ascontiguousarray(x)
    item = x.dtype.itemsize
    raw = np.empty(x.size + 128 // item, dtype=x.dtype)
    base = raw.ctypes.data
    start = (-base) % 64 // item + (0 if aligned else 1)
    out = raw[start:start + x.size]
    out[...] = x.ravel()
    return out


def ref_mtsv(a, b, c, d, u=None, solvedim=0, dims=None, pads=None, inc=False, threads=None):
    """Run the reference's tridS/DmtsvStridedBatch[Inc] (trid_cpu.cpp:535-595).

    The reference assumes exactly three dimensions (trid_cpu.cpp:406-531);
    shorter shapes are padded with 1s as scalar/test/test_cpu.cpp:96-98 does.
    solvedim 0 is routed through the correct scalar path by misaligned
    pointers; solvedim 1/2 need pads[0] to be a multiple of the SIMD width.
    """
    dims = [int(v) for v in dims]
    pads = dims if pads is None else [int(v) for v in pads]
    assert len(dims) <= 3
    dims3 = dims + [1] * (3 - len(dims))
    pads3 = pads + [1] * (3 - len(pads))
    dt = np.asarray(d).dtype
    simd = 4 if dt == np.float64 else 8
    if solvedim > 0 and pads3[0] % simd != 0:
        raise ValueError("reference y/z path needs pads[0] % SIMD_VEC == 0")
    aligned = solvedim > 0
    aa, bb, cc, dd = (_placed(x, aligned) for x in (a, b, c, d))
    uu = _placed(u, aligned) if inc else None
    name = ("tridD" if dt == np.float64 else "tridS") + "mtsvStridedBatch" + ("Inc" if inc else "")
    f = getattr(ref_lib(), name)
    f.restype = c_int
    st = f(_p(aa), _p(bb), _p(cc), _p(dd), _p(uu), c_int(3), c_int(solvedim), _ipad(dims3),
           _ipad(pads3))
    assert st == 0
    return np.array(uu if inc else dd, copy=True)


def ref_trid_scalar(a, b, c, d, n, stride):
    d = np.array(d, copy=True)
    f = ref_lib().trid_scalarD if d.dtype == np.float64 else ref_lib().trid_scalarS
    f(_p(a), _p(b), _p(c), _p(d), None, c_int(n), c_int(stride))
    return d


def ref_btsv_system_major(A, B, C, d, N, P, M):
    """The reference's block CPU gold dbtsv_cpu (blktrid_cpu.cpp:548-584),
    system-major layout, as shipped (including its matrix-product defect)."""
    A, B, C, d = (np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, C, d))
    Cs = np.zeros_like(C)
    ds = np.zeros_like(d)
    u = np.zeros_like(d)
    f = getattr(ref_block_lib(), "_Z9dbtsv_cpuPdS_S_S_S_S_S_iii")
    f(_p(A), _p(B), _p(C), _p(Cs), _p(ds), _p(d), _p(u), c_int(N), c_int(P), c_int(M))
    return u


def run_adi_orig(nx, ny, nz, iters, workdir):
    """Run the reference's sequential ADI gold program; returns u (x fastest)."""
    exe = os.path.join(HERE, "_ref", "adi_orig")
    link = os.path.join(workdir, "adi_orig")
    if not os.path.exists(link):
        os.symlink(exe, link)
    subprocess.run([link, "-nx", str(nx), "-ny", str(ny), "-nz", str(nz), "-iter", str(iters),
                    "-prof", "0"], check=True, capture_output=True, cwd=workdir)
    return np.fromfile(link + ".dat", dtype=np.float64)


# --------------------------------------------------------------------------- #
# Dense FP64 LU oracle (numpy)                                                #
# --------------------------------------------------------------------------- #
def dense_solve_systems(a, b, c, d):
    """Solve each row-system (shape [S, n]) by dense FP64 LU (numpy.linalg);
    complex inputs in complex128."""
    cplx = any(np.iscomplexobj(x) for x in (a, b, c, d))
    t = np.complex128 if cplx else np.float64
    a, b, c, d = (np.asarray(x, dtype=t) for x in (a, b, c, d))
    S, n = b.shape
    M = np.zeros((S, n, n), dtype=t)
    idx = np.arange(n)
    M[:, idx, idx] = b
    if n > 1:
        M[:, idx[1:], idx[:-1]] = a[:, 1:]
        M[:, idx[:-1], idx[1:]] = c[:, :-1]
    return np.linalg.solve(M, d[..., None])[..., 0]


def systems_view(x, dims, solvedim, pads=None):
    """Gather the systems of an N-D array (dims[0] fastest) as rows [S, n]."""
    dims = list(dims)
    pads = dims if pads is None else list(pads)
    cube = np.asarray(x).reshape(pads[::-1])  # C-order: last axis = dims[0]
    sl = tuple(slice(0, dims[k]) for k in range(len(dims)))[::-1]
    cube = cube[sl]
    ax = len(dims) - 1 - solvedim
    return np.moveaxis(cube, ax, -1).reshape(-1, dims[solvedim])
