"""Independent shards of a strided batch across ranks (one process per GPU).

The systems of a strided batch are independent, so N ranks split them with no
data exchange: each rank takes a contiguous range of the outermost non-solve
axis and solves that sub-batch with the ordinary entry points (its arrays
start at an element offset; dims carry the local extent; pads are unchanged,
since they also set the strides of the axes above).  The only collective is
the maximum over ranks of a measured time (or any scalar), which `bench.py
--gpus N` uses for its whole-job timing.
"""

from math import prod

__all__ = ["shard_range", "shard_batch", "max_over_ranks"]


def shard_range(n, rank, world):
    """Balanced contiguous split of range(n): this rank's [lo, hi)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need 0 <= rank < world and n >= 0")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_batch(dims, pads, solvedim, rank, world):
    """This rank's share of a strided batch (reference layout: element
    (i0, i1, ...) at i0 + pads[0]*(i1 + pads[1]*(...))).  Returns
    (element_offset, local_dims): the arrays of the share start element_offset
    elements in, and local_dims equals dims except on the outermost non-solve
    axis, which is split by shard_range."""
    dims, pads = list(dims), list(pads)
    nd = len(dims)
    if len(pads) < nd or not 0 <= solvedim < nd:
        raise ValueError("dims/pads/solvedim mismatch")
    axes = [i for i in range(nd) if i != solvedim]
    if not axes:
        raise ValueError("a single system (no non-solve axis) cannot be sharded")
    k = axes[-1]
    lo, hi = shard_range(dims[k], rank, world)
    local = list(dims)
    local[k] = hi - lo
    return lo * prod(pads[:k]), local


def max_over_ranks(value):
    """max of a scalar over the ranks of the default process group (the value
    itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
