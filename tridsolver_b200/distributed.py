"""Distributed strided-batch solve: every system split along the solve
dimension over the ranks of a process group.

The reference's MPI/NCCL build links the same four strided-batch entry
points and reads its distributed parameters from ``ctx.mpi_params``
(scalar/src/cuda/trid_cuda_mpi.cu:609-817, scalar/include/
trid_mpi_solver_params.hpp:47-181). Here ``DistContext`` registers a
``tridDistParams`` with the library and hands out a ``TridParams`` whose
``mpi_params`` points at it, so the ordinary calls

    tridDmtsvStridedBatch(dc.ctx, a, b, c, d, ndim, solvedim, dims, pads)

(or ``strided_batch(..., ctx=dc.ctx)``) run the partition method across
ranks. The library reduces every local segment to two boundary rows; the
exchange between its kernels is the allgather callback, by default
``torch.distributed.all_gather_into_tensor`` on the context's group (NCCL
over NVLink / NVSwitch between GPUs), which is ordered on torch's current
stream like any collective.

Each rank passes its own block: ``dims[solvedim]`` is its row count (at
least 2) and the other dimensions are the same on every rank.
"""

import ctypes

import torch

from . import _lib, api

ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                ctypes.c_void_p, ctypes.c_void_p)


class DistParams(ctypes.Structure):
    """struct tridDistParams (include/tridsolver_b200.h)."""
    _fields_ = [("solvedim", ctypes.c_int),
                ("rank", ctypes.c_int),
                ("nranks", ctypes.c_int),
                ("allgather", ALLGATHER_FN),
                ("user", ctypes.c_void_p)]


class _DeviceBytes:
    """A device buffer given by address and size, seen by torch as uint8."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3,
                                         "stream": None}


def device_bytes(ptr, nbytes, device):
    """Zero-copy uint8 tensor over nbytes of device memory at ptr."""
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


def torch_allgather(group):
    """Exchange over a torch.distributed group: gathers nbytes from every
    rank's send buffer into recv in rank order (one all_gather_into_tensor)."""
    import torch.distributed as dist

    def gather(send, recv, nbytes, nranks):
        dev = torch.device("cuda", torch.cuda.current_device())
        s = device_bytes(send, nbytes, dev)
        r = device_bytes(recv, nbytes * nranks, dev)
        dist.all_gather_into_tensor(r, s, group=group)

    return gather


class DistContext:
    """Distributed-solve parameters for solves along `solvedim`.

    rank / nranks default to the group's; `allgather(send_ptr, recv_ptr,
    nbytes, nranks)` replaces the torch.distributed exchange (the GPU tests
    use it to run several ranks as threads of one process). An exception in
    the exchange makes the solve fail and is re-raised from ``check``/the
    ``strided_batch`` wrapper."""

    def __init__(self, solvedim, group=None, rank=None, nranks=None, allgather=None):
        if rank is None or nranks is None:
            import torch.distributed as dist
            rank = dist.get_rank(group) if rank is None else rank
            nranks = dist.get_world_size(group) if nranks is None else nranks
        self.solvedim = int(solvedim)
        self.rank = int(rank)
        self.nranks = int(nranks)
        self._gather = allgather if allgather is not None else torch_allgather(group)
        self.error = None

        def cb(send, recv, nbytes, user, stream):
            try:
                self._gather(send, recv, nbytes, self.nranks)
                return 0
            except BaseException as e:  # reported after the library call returns
                self.error = e
                return 1

        self._cb = ALLGATHER_FN(cb)
        self._params = DistParams()
        lib = _lib.load()
        st = lib.tridDistInit(ctypes.addressof(self._params), self.solvedim, self.rank, self.nranks,
                              ctypes.cast(self._cb, ctypes.c_void_p), None)
        if st != 0:
            raise api.TridError(st, "tridDistInit")
        self.ctx = api.TridParams()
        self.ctx.mpi_params = ctypes.addressof(self._params)
        self._open = True

    def close(self):
        if self._open:
            _lib.load().tridDistFinalize(ctypes.addressof(self._params))
            self._open = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self):
        """Raises the exchange's exception, if the last solve's exchange failed."""
        if self.error is not None:
            e, self.error = self.error, None
            raise RuntimeError("distributed exchange failed") from e

    def exchange_bytes(self, dtype_bytes, dims):
        """Bytes this rank contributes per solve (6 values per system)."""
        return _lib.load().tridDistExchangeBytes(int(dtype_bytes), len(dims), self.solvedim,
                                                 api._ints(dims))

    def strided_batch(self, a, b, c, d, dims, pads=None, u=None):
        """This rank's block of a distributed solve along the context's
        dimension (tensors as for api.strided_batch); d <- x or u += x."""
        try:
            api.strided_batch(a, b, c, d, self.solvedim, dims, pads, u=u, ctx=self.ctx)
        except api.TridError:
            self.check()
            raise
        self.check()
