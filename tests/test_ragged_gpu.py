"""GPU: ragged batches in one persistent launch (tridDmtsvRaggedBatch).

Each system is checked against the oracle's per-system Thomas solve
(oracle_ragged_*, the reference's trid_scalar, scalar/src/cpu/
trid_cpu.cpp:312-353): normwise <= 1e-12 (FP64) / 1e-5 (FP32), per system
and over the batch. Lengths cover every path: empty and one-row systems,
pure PCR (<= 32), the warp hybrid for short classes, single tiles (512
rows) and systems of 2 to 32 tiles coupled through the second-level solve
(tile boundaries at every offset), up to the 16384-row limit, in shuffled
order.
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from oracle.pyoracle import Restatement

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


def _batch(lengths, dt, seed):
    rng = np.random.default_rng(seed)
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    n = int(offs[-1])
    a = rng.uniform(-0.5, 0.5, n)
    c = rng.uniform(-0.5, 0.5, n)
    b = 1 + np.abs(a) + np.abs(c) + rng.uniform(0, 1, n)
    d = rng.standard_normal(n)
    return [v.astype(dt) for v in (a, b, c, d)], offs


def _run(arrs, offs, dt):
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in arrs)
    to = torch.from_numpy(offs).cuda()
    fn = tb.tridDmtsvRaggedBatch if dt == np.float64 else tb.tridSmtsvRaggedBatch
    st = fn(None, ta, tb_, tc, td, to, len(offs) - 1)
    torch.cuda.synchronize()
    return st, td.cpu().numpy()


EDGE = [0, 1, 2, 3, 7, 8, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513,
        1000, 1023, 1024, 1025, 2048, 4095, 4096, 4097, 8191, 8192, 8193, 12000, 16383, 16384]


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_edge_lengths(dt, tol, oracle):
    lengths = np.array(EDGE * 3)
    np.random.default_rng(3).shuffle(lengths)
    arrs, offs = _batch(lengths, dt, seed=1)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    st, got = _run(arrs, offs, dt)
    assert st == 0
    for k in range(len(lengths)):
        s, e = offs[k], offs[k + 1]
        if e > s:
            den = np.max(np.abs(want[s:e]))
            err = np.max(np.abs(got[s:e].astype(np.float64) - want[s:e])) / den
            assert err <= tol, (k, e - s, err)


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_log_uniform_lengths(dt, tol, oracle):
    rng = np.random.default_rng(7)
    lengths = np.floor(np.exp(rng.uniform(np.log(8), np.log(16384), 3000))).astype(np.int64)
    arrs, offs = _batch(lengths, dt, seed=2)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    st, got = _run(arrs, offs, dt)
    assert st == 0
    err = np.max(np.abs(got.astype(np.float64) - want)) / np.max(np.abs(want))
    assert err <= tol


def test_autotune_then_solve(oracle):
    tb.ragged_autotune(8)
    table = tb.ragged_table(8)
    for cls, m in enumerate(table):
        assert m == 0 or 32 * m >= 2 ** cls  # 0: tiles; else the class fits its warp
    lengths = np.array([5, 40, 100, 300, 500, 60, 17] * 20)
    arrs, offs = _batch(lengths, np.float64, seed=4)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    st, got = _run(arrs, offs, np.float64)
    assert st == 0
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) <= 1e-12


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_too_long_system_is_reported(dt):
    arrs, offs = _batch(np.array([100, 16385, 7]), dt, seed=5)
    st, got = _run(arrs, offs, dt)
    assert st == tb.TridStatus.MATRIX_TYPE_NOT_SUPPORTED


def test_release_scratch_between_calls(oracle):
    """tridReleaseScratch hands the scratch pool's unused memory back to the
    driver; the next call refills the pool and gives the same result."""
    lengths = np.array([40, 700, 5000, 3, 1500] * 40)
    arrs, offs = _batch(lengths, np.float64, seed=6)
    st, first = _run(arrs, offs, np.float64)
    assert st == 0
    tb.release_scratch()
    tb.release_scratch()
    st, second = _run(arrs, offs, np.float64)
    assert st == 0
    assert np.array_equal(first, second)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    assert np.max(np.abs(second - want)) / np.max(np.abs(want)) <= 1e-12


def test_bounded_wait_runs_out_and_is_reported(oracle):
    """Failure detection without a GPU fault: the warp that solves each
    multi-tile system's second-level system withholds its publication (a
    flag that nothing sets), so the other tiles' bounded waits run out. The
    blocking call returns an error status, and the context stays usable: the
    same batch then solves normally."""
    lib = tb.load_library()
    lengths = np.array([3000, 40, 9000, 700, 2048] * 8)  # multi-tile in both precisions
    for dt in (np.float64, np.float32):
        arrs, offs = _batch(lengths, dt, seed=8)
        lib.tridRaggedSetWaitBound(1 << 14, 1)  # about 2 ms per wait
        try:
            st, _ = _run(arrs, offs, dt)
        finally:
            lib.tridRaggedSetWaitBound(0, 0)
        assert st == tb.TridStatus.EXECUTION_FAILED
        st, got = _run(arrs, offs, dt)
        assert st == 0
        want = arrs[3].copy()
        oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
        tol = 1e-12 if dt == np.float64 else 1e-5
        assert np.max(np.abs(got.astype(np.float64) - want)) / np.max(np.abs(want)) <= tol


def _sized(dt):
    return tb.tridDmtsvRaggedBatchSized if dt == np.float64 else tb.tridSmtsvRaggedBatchSized


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_sized_call_matches_the_counted_one(dt, tol, oracle):
    """tridDmtsvRaggedBatchSized with the exact element count, and with a
    larger one, gives the counted call's result bit for bit (the same
    kernels; only the scratch sizing differs), and the oracle's."""
    lengths = np.array(EDGE * 2)
    np.random.default_rng(9).shuffle(lengths)
    arrs, offs = _batch(lengths, dt, seed=10)
    st, first = _run(arrs, offs, dt)
    assert st == 0
    for nelems in (int(offs[-1]), int(offs[-1]) + 12345):
        ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in arrs)
        st = _sized(dt)(None, ta, tb_, tc, td, torch.from_numpy(offs).cuda(), len(lengths), nelems)
        torch.cuda.synchronize()
        assert st == 0
        assert np.array_equal(td.cpu().numpy(), first)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    assert np.max(np.abs(first.astype(np.float64) - want)) / np.max(np.abs(want)) <= tol


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_sized_call_refuses_a_short_count(dt):
    """A count below offsets[nsys] - offsets[0] is refused on the device
    before anything is written: d keeps its values, the blocking call returns
    INVALID_VALUE, and a negative count is refused on the host."""
    lengths = np.array([3000, 40, 9000, 700, 2048, 5] * 8)
    arrs, offs = _batch(lengths, dt, seed=11)
    total = int(offs[-1])
    to = torch.from_numpy(offs).cuda()
    for nelems in (total - 1, total // 4, 0):
        ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in arrs)
        st = _sized(dt)(None, ta, tb_, tc, td, to, len(lengths), nelems)
        torch.cuda.synchronize()
        assert st == tb.TridStatus.INVALID_VALUE, nelems
        assert np.array_equal(td.cpu().numpy(), arrs[3])
    st = _sized(dt)(None, ta, tb_, tc, td, to, len(lengths), -1)
    assert st == tb.TridStatus.INVALID_VALUE


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_sized_call_replays_in_a_cuda_graph(dt, tol, oracle):
    """The sized call, non-blocking, captured into a CUDA graph after one
    eager call: each replay copies the current right-hand side into d and
    solves it (the scratch is the graph's own allocation), and matches the
    oracle for three different right-hand sides."""
    lengths = np.array([1, 31, 33, 200, 513, 1025, 3000, 9000, 16384, 64] * 6)
    arrs, offs = _batch(lengths, dt, seed=12)
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in arrs)
    rhs = td.clone()
    to = torch.from_numpy(offs).cuda()
    nelems = int(offs[-1])

    def launch():
        td.copy_(rhs)
        st = _sized(dt)(None, ta, tb_, tc, td, to, len(lengths), nelems)
        assert st == 0

    with tb.on_stream(blocking=False):
        launch()
    torch.cuda.synchronize()
    tb.pivot_status()  # clears the record
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            with tb.on_stream(s, blocking=False):
                launch()
    torch.cuda.current_stream().wait_stream(s)
    rng = np.random.default_rng(13)
    for rep in range(3):
        d0 = rng.standard_normal(nelems).astype(dt)
        rhs.copy_(torch.from_numpy(d0))
        g.replay()
        torch.cuda.synchronize()
        want = d0.copy()
        oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
        got = td.cpu().numpy().astype(np.float64)
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) <= tol, rep
    assert tb.pivot_status() == tb.TridStatus.SUCCESS
    del g


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_bench_batch_of_200000_systems(dt, tol, oracle):
    """The benchmark's ragged batch itself: 200,000 systems with lengths
    floor(exp(U(ln 8, ln 16384))) (seed 0), about 4.3e8 elements, against
    the oracle's per-system solve, over the batch and per system."""
    rng = np.random.default_rng(0)
    lengths = np.floor(np.exp(rng.uniform(np.log(8), np.log(16384), 200000))).astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    n = int(offs[-1])
    g = torch.Generator(device="cuda").manual_seed(12)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    ta = torch.rand(n, generator=g, device="cuda", dtype=tdt) - 0.5
    tc = torch.rand(n, generator=g, device="cuda", dtype=tdt) - 0.5
    tb_ = 1 + ta.abs() + tc.abs() + torch.rand(n, generator=g, device="cuda", dtype=tdt)
    td = torch.randn(n, generator=g, device="cuda", dtype=tdt)
    a, b, c, want = (t.cpu().numpy() for t in (ta, tb_, tc, td))
    fn = tb.tridDmtsvRaggedBatch if dt == np.float64 else tb.tridSmtsvRaggedBatch
    st = fn(None, ta, tb_, tc, td, torch.from_numpy(offs).cuda(), len(lengths))
    torch.cuda.synchronize()
    assert st == 0
    del ta, tb_, tc
    got = td.cpu().numpy()
    del td
    torch.cuda.empty_cache()
    oracle.ragged(a, b, c, want, offs)
    del a, b, c
    diff = np.abs(got.astype(np.float64) - want)
    assert diff.max() / np.abs(want).max() <= tol
    # per system: the largest error relative to that system's own max |x|
    smax = np.maximum.reduceat(np.abs(want), offs[:-1])
    dmax = np.maximum.reduceat(diff, offs[:-1])
    assert np.max(dmax / smax) <= 10 * tol



@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
@pytest.mark.parametrize("lead", [1, 2, 3, 5])
def test_systems_at_every_alignment(dt, tol, lead, oracle):
    """Systems starting at every element offset modulo 16 bytes (the lead
    system's length shifts the rest), with lengths at and around tile
    multiples up to the 16384-row limit: tiles that start on a 16-byte
    boundary stage in 16-byte units, the others element by element, and
    every system matches the oracle."""
    lengths = np.array([lead, 16384, 510, 511, 512, 513, 1022, 1023, 1024, 1025, 16381, 3, 16384,
                        16383, 700, 1, 2047, 16382])
    arrs, offs = _batch(lengths, dt, seed=20 + lead)
    want = arrs[3].copy()
    oracle.ragged(arrs[0], arrs[1], arrs[2], want, offs)
    st, got = _run(arrs, offs, dt)
    assert st == 0
    for k in range(len(lengths)):
        s, e = offs[k], offs[k + 1]
        den = np.max(np.abs(want[s:e]))
        err = np.max(np.abs(got[s:e].astype(np.float64) - want[s:e])) / den
        assert err <= tol, (k, e - s, s % 4, err)
