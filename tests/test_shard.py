"""Sharding a strided batch across ranks (CPU, two gloo ranks).

The path shards with no exchange: each rank solves a contiguous range of the
outermost non-solve axis.  Checked here without a GPU: the shards of several
layouts cover every system exactly once (element offsets and local dims
turned back into system indices), and the one collective, the maximum of a
timing over ranks, returns the slowest rank's value on every rank.
"""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from tridsolver_b200.shard import max_over_ranks, shard_batch, shard_range  # noqa: E402

LAYOUTS = [([8, 5, 3], [8, 5, 3], 0), ([7, 9, 4], [10, 9, 4], 1), ([6, 4, 11], [6, 5, 11], 2),
           ([33, 2], [40, 2], 0), ([5, 3, 2, 7], [5, 3, 2, 7], 3)]


def systems_of(offset, local, dims, pads, solvedim):
    """System start offsets covered by a share (reference layout)."""
    strides = [int(np.prod(pads[:i])) for i in range(len(dims))]
    axes = [i for i in range(len(dims)) if i != solvedim]
    starts = set()
    for idx in np.ndindex(*[local[i] for i in axes]):
        starts.add(offset + sum(j * strides[i] for j, i in zip(idx, axes)))
    return starts


def test_shard_range_balanced():
    for n in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shares = [shard_batch(d, p, sd, rank, world) for d, p, sd in LAYOUTS]
        gathered = [None] * world
        dist.all_gather_object(gathered, shares)
        slowest = max_over_ranks(1.5 + rank)  # a per-rank "time"
        if rank == 0:
            out.put(("shares", gathered))
        out.put(("max", rank, slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_cover_every_system_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    msgs = [q.get(timeout=120) for _ in range(world + 1)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = next(m[1] for m in msgs if m[0] == "shares")
    for li, (dims, pads, sd) in enumerate(LAYOUTS):
        full = systems_of(0, dims, dims, pads, sd)
        seen = []
        for r in range(world):
            off, local = gathered[r][li]
            seen.extend(systems_of(off, local, dims, pads, sd))
        assert sorted(seen) == sorted(full), (dims, sd)
    maxes = [m[2] for m in msgs if m[0] == "max"]
    assert maxes == [2.5, 2.5]


GPU_LAYOUTS = [([256, 48, 40], [256, 48, 40], 0), ([64, 300, 20], [70, 300, 20], 1),
               ([40, 24, 257], [40, 24, 257], 2), ([1000, 37], [1024, 37], 0)]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_solve_matches_whole_batch(dtype, world):
    """Each rank's share, solved through the C ABI at its element offset with
    local dims (pads unchanged), reproduces the whole-batch solve: the shards
    of `world` ranks are solved here one after another on one GPU."""
    import tridsolver_b200 as tb

    tdt = getattr(torch, dtype)
    fn = tb.tridDmtsvStridedBatch if dtype == "float64" else tb.tridSmtsvStridedBatch
    tol = 1e-12 if dtype == "float64" else 1e-5
    gen = torch.Generator().manual_seed(7)
    for dims, pads, sd in GPU_LAYOUTS:
        size = int(np.prod(pads))
        a = (torch.rand(size, generator=gen, dtype=torch.float64) - 0.5).to(tdt).cuda()
        c = (torch.rand(size, generator=gen, dtype=torch.float64) - 0.5).to(tdt).cuda()
        b = (2.5 + torch.rand(size, generator=gen, dtype=torch.float64)).to(tdt).cuda()
        d = torch.randn(size, generator=gen, dtype=torch.float64).to(tdt).cuda()
        whole = d.clone()
        assert fn(a, b, c, whole, None, len(dims), sd, dims, pads) == 0
        shards = d.clone()
        for rank in range(world):
            off, local = shard_batch(dims, pads, sd, rank, world)
            if 0 in local:
                continue
            views = [t[off:] for t in (a, b, c, shards)]
            assert fn(*views, None, len(dims), sd, local, pads) == 0
        torch.cuda.synchronize()
        err = (shards - whole).abs().max().item() / max(whole.abs().max().item(), 1e-300)
        assert err <= tol, (dims, sd, err)
