"""Dependent solves back to back on one stream (GPU).

The axis-0, strided and ADI kernels are launched so that a kernel may be
scheduled while its predecessor on the stream drains; each must still read
its input only after that predecessor has finished writing it.  These tests
chain in-place solves (and torch kernels) with no host synchronisation in
between and compare the end result with the oracle applying the same steps
one after another."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402

from helpers import RTOL, rand_coeffs, rel_err  # noqa: E402


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("dims", [[256, 96, 80], [64, 48, 40]])
def test_in_place_solves_along_every_axis_back_to_back(dtype, dims):
    rng = np.random.default_rng(5)
    size = int(np.prod(dims))
    a, b, c, d = rand_coeffs(rng, size, dtype)
    # oracle: axis 0, then x * 2 - 1, then axis 1, then axis 2, then axis 0 again
    x = d.astype(np.float64)
    w = [v.astype(np.float64) for v in (a, b, c)]
    x = oracle.mtsv(*w, x, dims=dims, solvedim=0)
    x = x * 2 - 1
    x = oracle.mtsv(*w, x, dims=dims, solvedim=1)
    x = oracle.mtsv(*w, x, dims=dims, solvedim=2)
    x = oracle.mtsv(*w, x, dims=dims, solvedim=0)
    fn = tb.tridDmtsvStridedBatch if dtype == np.float64 else tb.tridSmtsvStridedBatch
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in (a, b, c, d))
    torch.cuda.synchronize()
    for sd in (0, None, 1, 2, 0):
        if sd is None:
            td.mul_(2).sub_(1)  # a torch kernel between two solves
        else:
            assert fn(ta, tb_, tc, td, None, 3, sd, dims, dims) == 0
    got = td.cpu().numpy()
    assert rel_err(got, x) <= 10 * RTOL[dtype]


def test_repeated_solve_of_its_own_output():
    # each solve reads what the previous launch wrote: 20 in-place solves
    # along axis 1, then along axis 0, with no synchronisation
    dims = [128, 64, 32]
    rng = np.random.default_rng(6)
    a, b, c, d = rand_coeffs(rng, int(np.prod(dims)))
    x = d.copy()
    for sd in [1] * 20 + [0] * 20:
        x = oracle.mtsv(a, b, c, x, dims=dims, solvedim=sd)
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in (a, b, c, d))
    torch.cuda.synchronize()
    for sd in [1] * 20 + [0] * 20:
        assert tb.tridDmtsvStridedBatch(ta, tb_, tc, td, None, 3, sd, dims, dims) == 0
    assert rel_err(td.cpu().numpy(), x) <= 1e-11
