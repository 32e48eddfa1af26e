"""Drop-in check: the reference's own GPU callers, compiled unchanged against
the reference's own headers (scalar/include/trid_cuda.h, trid_common.h) and
linked to libtridb200_cudacompat.so instead of the reference GPU library
(oracle/Makefile targets _ref/test_cuda_ref and _ref/adi_cuda_ref).

* scalar/test/test_cuda.cu:40-137 -- the reference's Catch GPU test program:
  solveX/Y/Z on its golden fixtures, FP64 and FP32, its own tolerances
  (scalar/test/utils.hpp:14-17).  The fixtures are written to the files/
  layout the program reads (gen_testcases.write_testcase) from the
  committed tests/golden/*.npz, which hold exactly the values its MeshLoader
  parses.
* apps/adi/src/adi_cuda.cu:285-329 -- the reference ADI application (its
  preproc kernel, then x, y solves and the Inc z solve through the 11-argument
  API with opts and sync), compared with the reference's sequential gold
  program adi_orig.c on the same grid through the sum of u after the
  iterations, the figure the application prints.
"""

import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle import oracle  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")
TEST_PROG = os.path.join(REF, "test_cuda_ref")
ADI_PROG = os.path.join(REF, "adi_cuda_ref")

# the fixtures scalar/test/test_cuda.cu reads (4-D ones only when MAXDIM > 3,
# which the reference header sets to 3)
FIXTURES = ["two_dim_large_solve0", "two_dim_large_solve1", "three_dim_large_solve0",
            "three_dim_large_solve1", "three_dim_large_solve2"]


def write_fixture(name, dst):
    """One fixture in the text layout of gen_testcases.write_testcase: ndim and
    solvedim, the dims, then a, b, c, d, u (FP64 solution) and u (FP32
    solution), one array per line (dims[0] fastest)."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    lines = [f"{int(z['ndim'])} {int(z['solvedim'])}", " ".join(str(int(v)) for v in z["dims"])]
    for k in ("a", "b", "c", "d", "u", "u_float"):
        lines.append(" ".join(repr(float(v)) for v in z[k]))
    with open(os.path.join(dst, name), "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.mark.skipif(not os.path.exists(TEST_PROG), reason="oracle/_ref/test_cuda_ref not built")
def test_reference_gpu_test_program_passes_against_this_library(tmp_path):
    files = tmp_path / "files"
    files.mkdir()
    for name in FIXTURES:
        write_fixture(name, str(files))
    r = subprocess.run([TEST_PROG], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    assert "All tests passed" in out, out[-4000:]
    # every test case ran: 3 test cases x {double, float}
    m = re.search(r"All tests passed \((\d+) assertions? in (\d+) test cases?\)", out)
    assert m and int(m.group(2)) == 6, out[-2000:]


def _adi_sum(out):
    m = re.search(r"end h_u sum = ([-+0-9.eE]+)", out)
    assert m, out[-2000:]
    return float(m.group(1))


@pytest.mark.skipif(not os.path.exists(ADI_PROG), reason="oracle/_ref/adi_cuda_ref not built")
@pytest.mark.parametrize("n,iters,opt", [(64, 10, 0), (64, 10, 3), (100, 4, 0)])
def test_reference_adi_application_against_gold(tmp_path, n, iters, opt):
    r = subprocess.run([ADI_PROG, f"-nx={n}", f"-ny={n}", f"-nz={n}", f"-iter={iters}",
                        f"-optx={opt}", f"-opty={opt}", f"-optz={opt}", "-prof=0"],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    got = _adi_sum(out)  # printed with %lg: six significant digits
    gold = oracle.run_adi_orig(n, n, n, iters, str(tmp_path))
    expect = float(gold.sum())
    assert abs(got - expect) <= 1e-5 * abs(expect), (got, expect)
