"""Regenerate the golden fixtures from the reference's own fixture generator.

The reference's file-driven Catch2 tests (scalar/test/test_cpu.cpp:88-110,
scalar/test/test_cuda.cu:58-82) load text fixtures written by
scalar/test/gen_testcases.py:95-109.  Those files are not shipped with the
reference, so this script imports that generator from a checkout of the
reference (``--reference``, default ``$TRID_REFERENCE_DIR``), runs its ``main()``
exactly as shipped (numpy seed 1, same call order, so every fixture draws the
same random stream as the original), parses the text files the generator
wrote (column-major, values rounded to 15 / 6 decimals exactly as the
reference's ``MeshLoader`` sees them) and stores them as ``.npz`` archives next
to this script.

Size policy: fixtures up to 3-D are kept whole.  The 4-D fixtures (32^4) and
the reduced-system fixture (256x256) are cropped on the non-solve axes (the
systems along the solve axis are independent, so every kept system is exactly
the reference's system, with the reference's expected solution).

Run:  python tests/golden/gen_golden.py [--reference PATH]
"""

import argparse
import contextlib
import importlib.util
import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (file name written by gen_testcases.main(), crop extent on non-solve axes or None)
FIXTURES = [
    ("one_dim_small", None),
    ("one_dim_large", None),
    ("two_dim_small_solve0", None),
    ("two_dim_small_solve1", None),
    ("two_dim_large_solve0", None),
    ("two_dim_large_solve1", None),
    ("three_dim_large_solve0", None),
    ("three_dim_large_solve1", None),
    ("three_dim_large_solve2", None),
    ("four_dim_large_solve0", 4),
    ("four_dim_large_solve1", 4),
    ("four_dim_large_solve2", 4),
    ("four_dim_large_solve3", 4),
    ("reduced_test_small", 16),
]


def parse_fixture(path):
    """Parse one text fixture in the layout of gen_testcases.write_testcase."""
    with open(path) as f:
        lines = f.read().split("\n")
    ndim, solvedim = (int(v) for v in lines[0].split())
    dims = [int(v) for v in lines[1].split()]
    assert len(dims) == ndim
    arrays = []
    for k in range(6):
        vals = np.array([float(v) for v in lines[2 + k].split()], dtype=np.float64)
        assert vals.size == int(np.prod(dims))
        # column-major (Fortran) flattening == dims[0] fastest, which is the
        # library's memory layout (element (i0,i1,..) at i0 + d0*(i1 + d1*...)).
        arrays.append(vals)
    a, b, c, d, u, u_float = arrays
    return ndim, solvedim, dims, a, b, c, d, u, u_float


def crop(dims, solvedim, keep, arrays):
    shape_f = tuple(dims)
    sl = tuple(slice(None) if ax == solvedim else slice(0, keep) for ax in range(len(dims)))
    out = []
    for arr in arrays:
        cube = arr.reshape(shape_f, order="F")[sl]
        out.append(np.asfortranarray(cube).ravel(order="F"))
    new_dims = [dims[ax] if ax == solvedim else min(keep, dims[ax]) for ax in range(len(dims))]
    return new_dims, out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TRID_REFERENCE_DIR"),
                    help="reference checkout (default: $TRID_REFERENCE_DIR)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("name the reference checkout with --reference or TRID_REFERENCE_DIR")
    gen_path = os.path.join(args.reference, "scalar", "test", "gen_testcases.py")
    spec = importlib.util.spec_from_file_location("ref_gen_testcases", gen_path)
    mod = importlib.util.module_from_spec(spec)
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                spec.loader.exec_module(mod)  # seeds numpy with 1 at import
                mod.main()
        finally:
            os.chdir(cwd)
        for name, keep in FIXTURES:
            ndim, solvedim, dims, *arrays = parse_fixture(os.path.join(tmp, name))
            if keep is not None:
                dims, arrays = crop(dims, solvedim, keep, arrays)
            a, b, c, d, u, u_float = arrays
            np.savez_compressed(
                os.path.join(HERE, name + ".npz"),
                ndim=ndim, solvedim=solvedim, dims=np.array(dims, dtype=np.int32),
                a=a, b=b, c=c, d=d, u=u, u_float=u_float,
            )
            print(f"{name}: dims={dims} solvedim={solvedim}", file=sys.stderr)


if __name__ == "__main__":
    main()
