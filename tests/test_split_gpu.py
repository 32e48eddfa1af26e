"""Split solve on the GPU: systems cut along the solve dimension into slabs.

Ranks are emulated in one process first: each slab -- a view of the global
arrays at its element offset, local dims along the solve dimension, global
pads -- goes through tridDmtsvStridedBatchSplitReduce, the slabs' numbers are
stacked in rank order (what the all-gather delivers), and every slab is
finished with tridDmtsvStridedBatchSplitFinish; the assembled result must
match the oracle's solve of the whole systems (FP64 1e-12, FP32 1e-5).  The
last test runs the public entry point tridDmtsvStridedBatchMPI in two
processes sharing the GPU, exchanging over a gloo group.
"""

import ctypes
import os
import socket
from math import prod

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tridsolver_b200 as tb  # noqa: E402
from oracle import oracle  # noqa: E402
from tridsolver_b200 import _lib  # noqa: E402

from helpers import RTOL, dev, host, rand_coeffs, rel_err  # noqa: E402


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def split_case(dtype, dims, solvedim, cuts, pads=None, inc=False, seed=0):
    rng = np.random.default_rng(seed)
    pads = list(dims) if pads is None else pads
    size = int(np.prod(pads))
    a, b, c, d = rand_coeffs(rng, size, dtype)
    u = rng.standard_normal(size).astype(dtype)
    expect = oracle.mtsv(a, b, c, d, u, dims=dims, pads=pads, solvedim=solvedim, inc=inc)
    ta, tb_, tc, td, tu = (dev(x) for x in (a, b, c, d, u))
    L = tb.lib()
    pre = "tridDmtsvStridedBatch" if dtype == np.float64 else "tridSmtsvStridedBatch"
    reduce_, finish = getattr(L, pre + "SplitReduce"), getattr(L, pre + "SplitFinish")
    stride = int(np.prod(pads[:solvedim]))
    nsys = prod(dims) // dims[solvedim]
    P = len(cuts) - 1
    slabs = []
    for r in range(P):
        local = list(dims)
        local[solvedim] = cuts[r + 1] - cuts[r]
        slabs.append((cuts[r] * stride, local))
    bnds = []
    for off, local in slabs:
        bnd = torch.empty((6, nsys), dtype=torch.float64, device="cuda")
        st = reduce_(vp(ta[off:]), vp(tb_[off:]), vp(tc[off:]), vp(td[off:]), len(dims), solvedim,
                     _lib.int_array(local), _lib.int_array(pads), vp(bnd))
        assert st == 0
        bnds.append(bnd)
    allb = torch.stack(bnds).contiguous()
    for r, (off, local) in enumerate(slabs):
        st = finish(vp(ta[off:]), vp(tb_[off:]), vp(tc[off:]), vp(td[off:]),
                    vp(tu[off:]) if inc else None, len(dims), solvedim, _lib.int_array(local),
                    _lib.int_array(pads), vp(allb), P, r, 1 if inc else 0)
        assert st == 0
    got_d, got_u = host(td), host(tu)
    if inc:
        assert np.array_equal(got_d, d), "Inc must leave d as it was"
        got = got_u
    else:
        got = got_d
    mask = np.zeros(pads[::-1], dtype=bool)
    mask[tuple(slice(0, n) for n in dims[::-1])] = True
    err = rel_err(got.reshape(pads[::-1])[mask], expect.reshape(pads[::-1])[mask])
    assert err <= RTOL[dtype], err
    return err


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim,cuts", [
    ([37, 50], 1, [0, 25, 50]),
    ([37, 50], 1, [0, 2, 30, 50]),            # a slab of two rows
    ([64, 9, 40], 2, [0, 10, 20, 30, 40]),
    ([100, 7], 0, [0, 33, 66, 100]),          # unit-stride axis
    ([30, 20, 12], 0, [0, 12, 30]),
    ([30, 20, 12], 1, [0, 7, 14, 20]),
    ([16, 64], 1, list(range(0, 65, 4))),     # 16 slabs of 4 rows
    ([9, 5000], 1, [0, 1234, 5000]),          # long slabs (blocked partition)
    ([6000, 4], 0, [0, 2500, 6000]),          # long unit-stride slabs
])
def test_split_matches_whole(dtype, dims, solvedim, cuts):
    split_case(dtype, dims, solvedim, cuts, seed=sum(dims) + len(cuts))


@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
def test_split_padded_inc(solvedim, inc):
    dims, pads = [24, 18, 20], [27, 18, 22]
    n = dims[solvedim]
    split_case(np.float64, dims, solvedim, [0, n // 3, n // 2, n], pads=pads, inc=inc,
               seed=solvedim + 10 * inc)


def test_split_one_slab_is_the_plain_solve():
    split_case(np.float64, [40, 33], 1, [0, 33], seed=5)


def test_split_rejects_bad_arguments():
    L = tb.lib()
    t = torch.ones(64, dtype=torch.float64, device="cuda")
    bnd = torch.empty((6, 8), dtype=torch.float64, device="cuda")
    one_row = _lib.int_array([8, 1])
    ok = _lib.int_array([8, 8])
    assert L.tridDmtsvStridedBatchSplitReduce(vp(t), vp(t), vp(t), vp(t), 2, 1, one_row, ok,
                                              vp(bnd)) == 3
    assert L.tridDmtsvStridedBatchSplitReduce(vp(t), vp(t), vp(t), vp(t), 2, 1, ok, ok,
                                              None) == 3
    for nranks, rank in ((0, 0), (2, 2), (2, -1)):
        assert L.tridDmtsvStridedBatchSplitFinish(vp(t), vp(t), vp(t), vp(t), None, 2, 1, ok, ok,
                                                  vp(bnd), nranks, rank, 0) == 3


# ---------------------------------------------- two processes, one GPU --
def _mp_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from tridsolver_b200.mpi import MpiSolverParams, tridDmtsvStridedBatchMPI

        params = MpiSolverParams.cartesian([1, world])  # split along dimension 1
        n0, n1 = 21, 40
        rng = np.random.default_rng(77)
        a, b, c, d = (x.reshape(n1, n0) for x in rand_coeffs(rng, n0 * n1))
        lo, hi = rank * n1 // world, (rank + 1) * n1 // world
        loc = [torch.from_numpy(np.ascontiguousarray(x[lo:hi])).cuda() for x in (a, b, c, d)]
        st = tridDmtsvStridedBatchMPI(params, *loc, None, 2, 1, [n0, hi - lo], [n0, hi - lo])
        torch.cuda.synchronize()
        out.put((rank, st, lo, hi, loc[3].cpu().numpy()))
    finally:
        dist.destroy_process_group()


def test_split_two_processes_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    procs = [ctx.Process(target=_mp_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n0, n1 = 21, 40
    rng = np.random.default_rng(77)
    a, b, c, d = rand_coeffs(rng, n0 * n1)
    expect = oracle.mtsv(a, b, c, d, dims=[n0, n1], solvedim=1).reshape(n1, n0)
    got = np.zeros((n1, n0))
    for rank, st, lo, hi, x in res:
        assert st == 0
        got[lo:hi] = x
    assert rel_err(got, expect) <= RTOL[np.float64]
