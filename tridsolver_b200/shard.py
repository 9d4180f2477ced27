"""Sharding a strided batch across ranks (one process per GPU).

The systems of a strided batch are independent, so a batch shards across
ranks with no exchange at all. Rank r takes a contiguous slab of the
outermost dimension that does not run along the solve, and solves it with
the library on its own GPU. The slab is the same (pointer offset, dims,
pads) problem shape the C ABI takes, so no data moves between ranks. This is
"weak scaling" when every rank holds its own grid, as bench.py runs it, and
"strong scaling" when ranks split one grid.

Systems that themselves span ranks (a z-slab decomposition of a full ADI
step: x and y local, z across ranks) need an exchange instead: the
partition method of the reference's MPI/NCCL build
(`scalar/src/cuda/trid_cuda_mpi.cu:218-605`), an all-gather of 6 values per
system and rank, then a reduced solve. That is `tridsolver_b200.distributed`
(the library's distributed solve behind ctx->mpi_params), not this module.
"""


def outer_dim(ndim, solvedim):
    """The dimension whose slabs are split across ranks."""
    if ndim == 1:
        return None
    return ndim - 1 if solvedim != ndim - 1 else ndim - 2


def shard_range(n, rank, world):
    """Contiguous [start, stop) of n items for `rank` of `world` (balanced)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def local_problem(dims, pads, solvedim, rank, world):
    """(element offset, local dims) of this rank's slab; dims/pads as the C ABI.

    Returns (0, dims) for a single system (ndim = 1), which cannot be split
    without the distributed partition method."""
    dims = list(dims)
    od = outer_dim(len(dims), solvedim)
    if od is None:
        return 0, dims
    start, stop = shard_range(dims[od], rank, world)
    stride = 1
    for p in pads[:od]:
        stride *= p
    local = dims.copy()
    local[od] = stop - start
    return start * stride, local
