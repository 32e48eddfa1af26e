"""Axis-0 systems of 4097..65,536 rows: one thread-block cluster per system
(kern_xclu.cu, the default there), against the oracle; FP64 1e-12, FP32
1e-5.  Covers partial last CTAs, pads, Inc, one-CTA-sized tails, the cluster
limit (16 CTAs) and the blocked partition past it, and the forced blocked
partition at the same lengths for comparison."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402

from test_scalar_gpu import run_case  # noqa: E402


@pytest.fixture(autouse=True)
def _auto_method():
    tb.set_method(0)
    yield
    tb.set_method(0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [4097, 5000, 8191, 8192, 8193, 12345, 32768, 65536])
def test_cluster_lengths(dtype, n):
    run_case(np.random.default_rng(n), dtype, [n, 3], 0)


@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,pads", [([6000, 4], [6002, 4]), ([9000, 2, 3], [9001, 3, 3]),
                                       ([20480, 5], None)])
def test_cluster_pads_and_inc(inc, dims, pads):
    run_case(np.random.default_rng(len(dims) + inc), np.float64, dims, 0, pads=pads, inc=inc)


@pytest.mark.parametrize("n", [65537, 70000])
def test_past_the_cluster_limit_falls_back(n):
    run_case(np.random.default_rng(n), np.float64, [n, 2], 0)


@pytest.mark.parametrize("method", [(2, 8, 0), (2, 16, 0), (6, 16, 0)])
def test_forced_blocked_and_cluster_agree(method):
    run_case(np.random.default_rng(11), np.float64, [16384, 5], 0, method=method)
