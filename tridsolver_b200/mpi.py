"""Systems split along the solve dimension across ranks (one process per GPU).

The reference's distributed solve (scalar/include/trid_mpi_cuda.hpp:51-80,
scalar/include/trid_mpi_solver_params.hpp:48-140, implementation
scalar/src/cuda/trid_cuda_mpi.cu:473-583): every rank holds one slab of rows
of every system -- its local dims along the solve dimension -- and the ranks
along that dimension solve the full systems together.  Same entry points here
(``tridDmtsvStridedBatchMPI(params, a, b, c, d, u, ndim, solvedim, dims,
pads)`` and the Inc / FP32 forms, returning a tridStatus_t), over
torch.distributed instead of MPI:

  1. tridDmtsvStridedBatchSplitReduce (C ABI): the slab -> six numbers per
     system;
  2. an all-gather of those numbers over the process group of the solve
     dimension (NCCL over NVLink between GPUs; 48 bytes per system and rank,
     the reference's "6 reals per system per rank");
  3. tridDmtsvStridedBatchSplitFinish (C ABI): the slab solved from every
     rank's numbers.

Only the reference's ALLGATHER strategy exists (every rank combines the
gathered slabs itself); the other strategies and the mini-batch size are
accepted and ignored.  CUDA tensors throughout; a gloo group (CPU
collectives) gets host copies for the exchange.
"""

import ctypes
import itertools
from math import prod

from ._lib import int_array, lib
from .scalar import _bind_stream, _ptr

__all__ = ["MpiSolverParams", "tridDmtsvStridedBatchMPI", "tridSmtsvStridedBatchMPI",
           "tridDmtsvStridedBatchIncMPI", "tridSmtsvStridedBatchIncMPI", "gather_slabs"]

GATHER_SCATTER, ALLGATHER, LATENCY_HIDING_INTERLEAVED, LATENCY_HIDING_TWO_STEP = range(4)


class MpiSolverParams:
    """Process layout of a split solve (trid_mpi_solver_params.hpp:48-140).

    num_procs[k]: ranks along dimension k; coords[k]: this rank's position
    along it; groups[k]: the torch.distributed process group of the ranks that
    share every other coordinate, holding them in the order of their
    coordinate along k (None for a dimension of one rank).
    """

    def __init__(self, num_procs, coords, groups, mpi_batch_size=32,
                 strategy=LATENCY_HIDING_INTERLEAVED):
        self.num_procs = [int(v) for v in num_procs]
        self.mpi_coords = [int(v) for v in coords]
        self.groups = list(groups)
        self.mpi_batch_size = int(mpi_batch_size)  # accepted, not used
        self.strategy = int(strategy)  # accepted: every strategy gathers on all ranks
        if not (len(self.num_procs) == len(self.mpi_coords) == len(self.groups)):
            raise ValueError("num_procs, coords and groups need one entry per dimension")

    @classmethod
    def cartesian(cls, num_procs, **kw):
        """The layout over the default process group, its ranks on a
        cartesian grid with dimension 0 fastest (rank = c0 + n0*(c1 + n1*...)),
        and one sub-group per grid line.  Collective: every rank calls it with
        the same num_procs."""
        import torch.distributed as dist

        num_procs = [int(v) for v in num_procs]
        world = dist.get_world_size()
        if prod(num_procs) != world:
            raise ValueError(f"grid {num_procs} needs {prod(num_procs)} ranks, have {world}")
        me = dist.get_rank()

        def coords_of(r):
            out = []
            for n in num_procs:
                out.append(r % n)
                r //= n
            return out

        def rank_of(cs):
            r, m = 0, 1
            for c, n in zip(cs, num_procs):
                r += c * m
                m *= n
            return r

        mine = coords_of(me)
        groups = []
        for k, n in enumerate(num_procs):
            mine_g = None
            others = [range(m) for j, m in enumerate(num_procs) if j != k]
            # every rank creates every group, in the same order
            for rest in itertools.product(*others):
                cs = list(rest)
                members = [rank_of(cs[:k] + [i] + cs[k:]) for i in range(n)]
                g = dist.new_group(members) if n > 1 else None
                if me in members:
                    mine_g = g
            groups.append(mine_g)
        return cls(num_procs, mine, groups, **kw)


def gather_slabs(bnd, group, nranks):
    """All-gather of one rank's [6, nsys] FP64 slab numbers over `group`, in
    rank order: [nranks, 6, nsys] on bnd's device."""
    import torch
    import torch.distributed as dist

    if nranks == 1 or group is None:
        return bnd.reshape(1, *bnd.shape)
    host = dist.get_backend(group) == "gloo" and bnd.is_cuda
    src = (bnd.cpu() if host else bnd).contiguous()
    # concatenated along dimension 0 (the form every backend takes), then split
    out = torch.empty((nranks * src.shape[0],) + tuple(src.shape[1:]), dtype=src.dtype,
                      device=src.device)
    dist.all_gather_into_tensor(out, src, group=group)
    out = out.reshape((nranks,) + tuple(src.shape))
    return out.to(bnd.device) if host else out


def _split_solve(prefix, inc, params, a, b, c, d, u, ndim, solvedim, dims, pads):
    import torch

    L = lib()
    _bind_stream(L)
    nsys = prod(int(dims[k]) for k in range(ndim) if k != solvedim)
    nranks = params.num_procs[solvedim]
    rank = params.mpi_coords[solvedim]
    group = params.groups[solvedim]
    dev = d.device if isinstance(d, torch.Tensor) else torch.device("cuda")
    bnd = torch.empty((6, max(nsys, 1)), dtype=torch.float64, device=dev)
    dims_c, pads_c = int_array(dims), int_array(pads)
    st = getattr(L, prefix + "SplitReduce")(_ptr(a), _ptr(b), _ptr(c), _ptr(d), ndim, solvedim,
                                            dims_c, pads_c, ctypes.c_void_p(bnd.data_ptr()))
    # every rank takes part in the exchange, whatever its status: a rank that
    # skipped it would leave the others waiting
    flag = torch.tensor([float(st)], dtype=torch.float64, device=dev)
    allb = gather_slabs(bnd, group, nranks)
    flags = gather_slabs(flag.reshape(1, 1), group, nranks)
    if st != 0:
        return st
    worst = int(flags.max().item())
    if worst != 0:
        return worst
    return getattr(L, prefix + "SplitFinish")(_ptr(a), _ptr(b), _ptr(c), _ptr(d),
                                              _ptr(u) if inc else None, ndim, solvedim, dims_c,
                                              pads_c, ctypes.c_void_p(allb.data_ptr()), nranks,
                                              rank, 1 if inc else 0)


def tridDmtsvStridedBatchMPI(params, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _split_solve("tridDmtsvStridedBatch", False, params, a, b, c, d, u, ndim, solvedim,
                        dims, pads)


def tridSmtsvStridedBatchMPI(params, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _split_solve("tridSmtsvStridedBatch", False, params, a, b, c, d, u, ndim, solvedim,
                        dims, pads)


def tridDmtsvStridedBatchIncMPI(params, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _split_solve("tridDmtsvStridedBatch", True, params, a, b, c, d, u, ndim, solvedim,
                        dims, pads)


def tridSmtsvStridedBatchIncMPI(params, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _split_solve("tridSmtsvStridedBatch", True, params, a, b, c, d, u, ndim, solvedim,
                        dims, pads)
