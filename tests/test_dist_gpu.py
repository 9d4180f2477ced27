"""GPU: the distributed solve (every system split along the solve dimension
over P ranks, the reference's MPI/NCCL partition method), run as P ranks in
threads of one process on one GPU.

Each thread is a rank with its own CUDA stream and its own DistContext; the
exchange between the library's kernels is a host-side all-gather among the
threads (a barrier and device copies), so no kernel ever waits on another.
The ranks' blocks are views of one global grid (dims = the rank's block,
pads = the global grid); the assembled result is compared with the oracle's
solve of the whole grid. Covers every solve dimension, 2 to 4 ranks, uneven
splits down to 2 rows per rank, Inc (u += x with d left unchanged), FP32,
and a failing exchange (reported as an error, without hanging).
"""

import threading

import numpy as np
import pytest
import torch

from helpers import make_system, normwise
from oracle.pyoracle import Restatement
from tridsolver_b200 import api
from tridsolver_b200.distributed import DistContext, device_bytes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


class ThreadExchange:
    """All-gather among threads: every rank publishes its send buffer, waits
    for the others, copies all of them into its receive buffer, and waits
    again before its send buffer may be released."""

    def __init__(self, nranks, timeout=60.0):
        self.barrier = threading.Barrier(nranks, timeout=timeout)
        self.slots = [None] * nranks

    def for_rank(self, rank):
        def gather(send, recv, nbytes, nranks):
            dev = torch.device("cuda", torch.cuda.current_device())
            torch.cuda.current_stream().synchronize()  # this rank's rows are written
            self.slots[rank] = device_bytes(send, nbytes, dev)
            self.barrier.wait()
            r = device_bytes(recv, nbytes * nranks, dev)
            for k in range(nranks):
                r[k * nbytes:(k + 1) * nbytes].copy_(self.slots[k])
            torch.cuda.current_stream().synchronize()
            self.barrier.wait()

        return gather


def run_ranks(nranks, fn):
    errors = [None] * nranks

    def worker(r):
        try:
            with torch.cuda.stream(torch.cuda.Stream()):
                fn(r)
                torch.cuda.current_stream().synchronize()
        except BaseException as e:  # noqa: BLE001 - collected and re-raised below
            errors[r] = e

    threads = [threading.Thread(target=worker, args=(r,)) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    return errors


def _stride(dims, sd):
    s = 1
    for i in range(sd):
        s *= dims[i]
    return s


def _solve_split(dims, sd, splits, dtype, inc, seed):
    a, b, c, d = [torch.from_numpy(v).cuda() for v in make_system(dims, sd, dtype, seed=seed)]
    u = torch.zeros_like(d) if inc else None
    d_in = d.clone()
    ex = ThreadExchange(len(splits))
    offs = np.concatenate([[0], np.cumsum(splits)])
    st = _stride(dims, sd)

    def rank_fn(r):
        local = list(dims)
        local[sd] = int(splits[r])
        base = int(offs[r]) * st
        with DistContext(sd, rank=r, nranks=len(splits), allgather=ex.for_rank(r)) as dc:
            dc.strided_batch(a[base:], b[base:], c[base:], d[base:], local, pads=dims,
                             u=None if u is None else u[base:])

    errors = run_ranks(len(splits), rank_fn)
    for e in errors:
        if e is not None:
            raise e
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (a, b, c, d_in)], d.cpu().numpy(), (None if u is None else u.cpu().numpy())


@pytest.mark.parametrize("dims,sd,splits", [
    ([12, 5, 7], 0, [6, 6]),
    ([7, 40, 6], 1, [10, 13, 17]),
    ([5, 6, 64], 2, [16, 16, 16, 16]),
    ([9, 4, 11], 2, [2, 7, 2]),
    ([33, 3, 2], 0, [2, 29, 2]),
    ([256, 8, 8], 0, [128, 128]),
    ([16, 16, 300], 2, [100, 150, 50]),
    # x segments of 32 M rows: the warp-tile reduction (M = 8, 16), beside
    # one that takes the lane-per-system reduction (64 rows)
    ([512, 6, 5], 0, [256, 256]),
    ([1024, 3, 4], 0, [512, 512]),
    ([320, 4, 3], 0, [256, 64]),
])
def test_distributed_f64(dims, sd, splits, oracle):
    (a, b, c, d0), x, _ = _solve_split(dims, sd, splits, np.float64, False, seed=sum(splits))
    ref = d0.copy()
    oracle.strided_batch(a, b, c, ref, dims, sd)
    assert normwise(x, ref) <= 1e-12


@pytest.mark.parametrize("dims,sd,splits", [([16, 24, 10], 1, [8, 16]), ([6, 5, 90], 2, [30, 30, 30]),
                                            ([512, 4, 3], 0, [128, 256, 128]),
                                            ([2048, 3, 2], 0, [1024, 1024])])
def test_distributed_f32(dims, sd, splits, oracle):
    (a, b, c, d0), x, _ = _solve_split(dims, sd, splits, np.float32, False, seed=3)
    ref = d0.astype(np.float64)
    oracle.strided_batch(a.astype(np.float64), b.astype(np.float64), c.astype(np.float64), ref, dims, sd)
    assert normwise(x, ref) <= 1e-5


@pytest.mark.parametrize("sd", [0, 1, 2])
def test_distributed_inc_leaves_d(sd, oracle):
    dims = [20, 18, 16]
    splits = {0: [10, 10], 1: [5, 6, 7], 2: [8, 4, 4]}[sd]
    (a, b, c, d0), d_after, u = _solve_split(dims, sd, splits, np.float64, True, seed=11)
    ref = d0.copy()
    oracle.strided_batch(a, b, c, ref, dims, sd)
    assert normwise(u, ref) <= 1e-12
    assert np.array_equal(d_after, d0)


def test_distributed_inc_tile_segments(oracle):
    """Inc through the warp-tile reduction (x segments of 256 rows)."""
    dims = [512, 5, 4]
    (a, b, c, d0), d_after, u = _solve_split(dims, 0, [256, 256], np.float64, True, seed=13)
    ref = d0.copy()
    oracle.strided_batch(a, b, c, ref, dims, 0)
    assert normwise(u, ref) <= 1e-12
    assert np.array_equal(d_after, d0)


def test_one_rank_is_the_ordinary_solve(oracle):
    (a, b, c, d0), x, _ = _solve_split([24, 10, 9], 1, [10], np.float64, False, seed=5)
    ref = d0.copy()
    oracle.strided_batch(a, b, c, ref, [24, 10, 9], 1)
    assert normwise(x, ref) <= 1e-12


def test_failed_exchange_is_reported():
    """Rank 1's exchange fails before it joins; rank 0's exchange gives up
    (the barrier is aborted) and both solves return an error; the GPU stays
    usable."""
    dims, sd, splits = [8, 6, 10], 2, [5, 5]
    a, b, c, d = [torch.from_numpy(v).cuda() for v in make_system(dims, sd, np.float64, seed=2)]
    ex = ThreadExchange(2, timeout=10.0)
    ok_gather = ex.for_rank(0)

    def failing(send, recv, nbytes, nranks):
        ex.barrier.abort()
        raise ConnectionError("rank 1 lost")

    def rank_fn(r):
        local = list(dims)
        local[sd] = splits[r]
        base = r * splits[0] * dims[0] * dims[1]
        with DistContext(sd, rank=r, nranks=2, allgather=ok_gather if r == 0 else failing) as dc:
            dc.strided_batch(a[base:], b[base:], c[base:], d[base:], local, pads=dims)

    errors = run_ranks(2, rank_fn)
    assert all(isinstance(e, RuntimeError) for e in errors), errors
    assert isinstance(errors[1].__cause__, ConnectionError)
    x = d.clone()
    api.strided_batch(a, b, c, x, sd, dims)
    torch.cuda.synchronize()
    assert torch.isfinite(x).all()


def test_unregistered_params_are_ignored(oracle):
    """An mpi_params that tridDistInit did not register (a stale or
    uninitialised pointer) is never dereferenced: the call is the ordinary
    single-GPU solve."""
    dims, sd = [10, 9, 8], 2
    a, b, c, d = [torch.from_numpy(v).cuda() for v in make_system(dims, sd, np.float64, seed=4)]
    ctx = api.TridParams()
    ctx.mpi_params = 0x1234
    want = d.cpu().numpy().copy()
    oracle.strided_batch(a.cpu().numpy(), b.cpu().numpy(), c.cpu().numpy(), want, dims, sd)
    api.strided_batch(a, b, c, d, sd, dims, ctx=ctx)
    torch.cuda.synchronize()
    assert normwise(d.cpu().numpy(), want) <= 1e-12
