"""Split solve host logic (CPU, gloo ranks): the process layout and the
exchange.

MpiSolverParams.cartesian puts the default group's ranks on a grid (axis 0
fastest) and gives every rank, per dimension, the group of its grid line;
gather_slabs all-gathers one rank's [6, nsys] slab numbers over that group
in the order of the coordinate along the dimension.  Checked with four gloo
ranks on a 2 x 2 grid: every line's gather comes back in coordinate order on
every rank of the line, and a dimension of one rank needs no group.
"""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _worker(rank, world, port, grid, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tridsolver_b200.mpi import MpiSolverParams, gather_slabs

        p = MpiSolverParams.cartesian(grid)
        res = {"coords": p.mpi_coords}
        for k in range(len(grid)):
            bnd = torch.full((6, 3), float(rank), dtype=torch.float64)
            got = gather_slabs(bnd, p.groups[k], p.num_procs[k])
            res[k] = [int(v) for v in got[:, 0, 0].tolist()]
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("grid", [[2, 2], [4, 1], [1, 4]])
def test_cartesian_groups_gather_in_coordinate_order(grid):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 4
    procs = [ctx.Process(target=_worker, args=(r, world, port, grid, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        c0, c1 = r % grid[0], r // grid[0]
        assert res[r]["coords"] == [c0, c1]
        # dimension 0: the ranks of this rank's row, by coordinate 0
        assert res[r][0] == [i + grid[0] * c1 for i in range(grid[0])]
        # dimension 1: the ranks of this rank's column, by coordinate 1
        assert res[r][1] == [c0 + grid[0] * j for j in range(grid[1])]
