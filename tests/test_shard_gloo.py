"""CPU: the multi-rank path (world size 2, gloo).

Each rank solves its slab of a batch (tridsolver_b200.shard.local_problem),
here with the CPU oracle standing in for the GPU solve, since the test is of
the sharding logic. Rank 0 gathers the slabs and compares them with the
whole batch solved at once. The ranks also reduce their timings with MAX,
as bench.py does, and exercise uneven splits, every solve dimension and a
padded layout.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tridsolver_b200.shard import local_problem, shard_range


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CASES = [([6, 5, 7], 0, None), ([6, 5, 7], 1, None), ([6, 5, 7], 2, None), ([9, 11], 0, None),
         ([9, 11], 1, None), ([5, 6, 3], 1, [7, 8, 3])]


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    from helpers import make_system
    from oracle.pyoracle import Restatement
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    oracle = Restatement()
    ok = True
    for dims, sd, pads in CASES:
        pads = pads or dims
        a, b, c, d = make_system(pads, sd, np.float64, seed=len(dims) + sd)
        off, ldims = local_problem(dims, pads, sd, rank, world)
        mine = d.copy()
        if int(np.prod(ldims)) > 0:
            oracle.strided_batch(a[off:], b[off:], c[off:], mine[off:], ldims, sd, pads=pads)
        # the slabs are disjoint: summing each rank's change reassembles the solve
        delta = torch.from_numpy(mine - d)
        dist.all_reduce(delta, op=dist.ReduceOp.SUM)
        if rank == 0:
            want = d.copy()
            oracle.strided_batch(a, b, c, want, dims, sd, pads=pads)
            got = d + delta.numpy()
            ok &= bool(np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want)))
    t = torch.tensor([float(rank + 1)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ok &= t.item() == float(world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ok))


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 8, 100):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(got[i][1] == got[i + 1][0] for i in range(world - 1))
            assert max(s - a for a, s in got) - min(s - a for a, s in got) <= 1


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results == {0: True, 1: True}
