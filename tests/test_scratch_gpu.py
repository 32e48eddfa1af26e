"""Library scratch across streams and CUDA graphs (GPU).

Long axis-0 systems (solved in blocks, the block rows in scratch) and the
variable-length batch (work tables in scratch) are run on several streams at
once and must match the same solves run one after another, bit for bit; a
CUDA graph captured on a stream that never made a call before, with problems
larger than anything solved eagerly, must replay to the eager results, and
keep doing so after tridReleaseScratch frees the buffers kept for eager
calls."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import tridsolver_b200 as tb  # noqa: E402
from tridsolver_b200.varlen import solve_varlen  # noqa: E402

from helpers import rand_coeffs  # noqa: E402


def long_problem(n, nsys, seed):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(x).cuda() for x in rand_coeffs(rng, n * nsys, np.float64)]


def varlen_problem(nsys, seed):
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(8192), nsys))).astype(np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    coeffs = [torch.from_numpy(x).cuda() for x in rand_coeffs(rng, int(off[-1]), np.float64)]
    return coeffs, torch.from_numpy(off).cuda()


def solve_long(p, n, nsys, x):
    a, b, c, _ = p
    tb.tridDmtsvStridedBatch(a, b, c, x, None, 2, 0, [n, nsys], [n, nsys])


def test_concurrent_streams_do_not_share_scratch():
    shapes = [(12000, 48), (20000, 40)]
    longs = [long_problem(n, s, 10 + k) for k, (n, s) in enumerate(shapes)]
    (vc, voff) = varlen_problem(1500, 20)
    # one after another on one stream
    ref = []
    for (n, s), p in zip(shapes, longs):
        x = p[3].clone()
        solve_long(p, n, s, x)
        ref.append(x)
    vref = vc[3].clone()
    solve_varlen(vc[0], vc[1], vc[2], vref, voff)
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in range(3)]
    reps = 12
    outs = [[None] * reps for _ in range(3)]
    for k in range(reps):
        for j, st in enumerate(streams):
            with torch.cuda.stream(st):
                if j < 2:
                    (n, s), p = shapes[j], longs[j]
                    x = p[3].clone()
                    solve_long(p, n, s, x)
                else:
                    x = vc[3].clone()
                    solve_varlen(vc[0], vc[1], vc[2], x, voff)
                outs[j][k] = x
    torch.cuda.synchronize()
    for j in range(3):
        want = ref[j] if j < 2 else vref
        for k in range(reps):
            assert torch.equal(outs[j][k], want), (j, k)


def test_graph_capture_allocates_in_stream_order():
    # lazy per-device setup (error word, kernel attributes) on the default
    # stream with problems smaller than the captured ones
    small = long_problem(5000, 2, 1)
    x = small[3].clone()
    solve_long(small, 5000, 2, x)
    (vsc, vsoff) = varlen_problem(10, 2)
    solve_varlen(vsc[0], vsc[1], vsc[2], vsc[3].clone(), vsoff)
    torch.cuda.synchronize()

    n, s = 16000, 64
    p = long_problem(n, s, 3)
    (vc, voff) = varlen_problem(2000, 4)
    want = p[3].clone()
    solve_long(p, n, s, want)
    vwant = vc[3].clone()
    solve_varlen(vc[0], vc[1], vc[2], vwant, voff)
    torch.cuda.synchronize()

    x = torch.empty_like(p[3])
    vx = torch.empty_like(vc[3])
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        x.copy_(p[3])
        solve_long(p, n, s, x)
        vx.copy_(vc[3])
        solve_varlen(vc[0], vc[1], vc[2], vx, voff)
    for _ in range(2):
        x.zero_()
        vx.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(x, want)
        assert torch.equal(vx, vwant)
    # the graph refers to none of the buffers kept for eager calls
    assert tb.lib().tridReleaseScratch() == 0
    x.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(x, want)
    del g


def test_release_then_solve_again():
    n, s = 9000, 8
    p = long_problem(n, s, 5)
    want = p[3].clone()
    solve_long(p, n, s, want)
    torch.cuda.synchronize()
    assert tb.lib().tridReleaseScratch() == 0
    x = p[3].clone()
    solve_long(p, n, s, x)
    torch.cuda.synchronize()
    assert torch.equal(x, want)
