"""CPU: host-side logic of the distributed solve (no GPU).

* tridDistInit / tridDistFinalize / tridDistExchangeBytes: argument checks,
  registration, exchange sizes (6 values per system and rank);
* the exchange plumbing of DistContext over a world-size-2 gloo group: the
  library's allgather callback, driven here with host buffers, gathers every
  rank's bytes in rank order;
* a rank that drops out before the exchange: the other rank's exchange ends
  with the process group's timeout, the callback reports the failure (the
  library would return TRID_STATUS_EXECUTION_FAILED) and DistContext.check
  raises, instead of anyone hanging.
"""

import ctypes
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tridsolver_b200 import _lib, api
from tridsolver_b200.distributed import DistContext, DistParams


def test_init_checks_and_registration():
    lib = _lib.load()
    p = DistParams()
    addr = ctypes.addressof(p)
    cb = ctypes.cast(ctypes.CFUNCTYPE(ctypes.c_int)(lambda: 0), ctypes.c_void_p)
    assert lib.tridDistInit(addr, 2, 1, 4, cb, None) == 0
    assert (p.solvedim, p.rank, p.nranks) == (2, 1, 4)
    assert lib.tridDistFinalize(addr) == 0
    assert lib.tridDistFinalize(addr) == api.TridStatus.INVALID_VALUE  # not registered any more
    for args in [(3, 0, 1), (0, 2, 2), (0, -1, 2), (0, 0, 0), (-1, 0, 1)]:
        assert lib.tridDistInit(addr, *args, cb, None) == api.TridStatus.INVALID_VALUE
    assert lib.tridDistInit(addr, 0, 0, 1, None, None) == api.TridStatus.INVALID_VALUE


def test_exchange_bytes():
    lib = _lib.load()
    dims = api._ints([10, 20, 30])
    assert lib.tridDistExchangeBytes(8, 3, 0, dims) == 6 * 20 * 30 * 8
    assert lib.tridDistExchangeBytes(4, 3, 2, dims) == 6 * 10 * 20 * 4
    assert lib.tridDistExchangeBytes(8, 2, 1, dims) == 6 * 10 * 8
    assert lib.tridDistExchangeBytes(2, 3, 0, dims) == -1
    assert lib.tridDistExchangeBytes(8, 3, 3, dims) == -1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _host_gather(group):
    """The exchange over gloo with host buffers (the library hands device
    buffers to its callback; this stands in for them on a CPU-only box)."""

    def gather(send, recv, nbytes, nranks):
        s = torch.frombuffer((ctypes.c_uint8 * nbytes).from_address(send), dtype=torch.uint8)
        r = torch.frombuffer((ctypes.c_uint8 * (nbytes * nranks)).from_address(recv), dtype=torch.uint8)
        parts = [torch.empty(nbytes, dtype=torch.uint8) for _ in range(nranks)]
        dist.all_gather(parts, s.clone(), group=group)
        r.copy_(torch.cat(parts))

    return gather


def _worker(rank, world, port, mode, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    try:
        dc = DistContext(2, allgather=_host_gather(None))
        assert (dc.rank, dc.nranks) == (rank, world)
        nbytes = 6 * 7 * 8
        send = np.full(nbytes, rank + 1, dtype=np.uint8)
        recv = np.zeros(nbytes * world, dtype=np.uint8)
        if mode == "drop" and rank == 1:
            q.put((rank, "dropped"))  # leaves without joining the exchange
            return
        rc = dc._cb(send.ctypes.data, recv.ctypes.data, nbytes, None, None)
        if mode == "ok":
            ok = rc == 0 and all((recv[k * nbytes:(k + 1) * nbytes] == k + 1).all() for k in range(world))
            q.put((rank, bool(ok)))
        else:
            try:
                dc.check()
                q.put((rank, "no error"))
            except RuntimeError:
                q.put((rank, "failed" if rc != 0 else "rc0"))
        dc.close()
    finally:
        if not (mode == "drop" and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


@pytest.mark.parametrize("mode", ["ok", "drop"])
def test_exchange_over_gloo(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    if mode == "ok":
        assert results == {0: True, 1: True}
    else:
        assert results == {0: "failed", 1: "dropped"}
