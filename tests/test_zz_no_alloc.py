"""GPU: tridDmtsvStridedBatchNoAlloc, the entry point for callers that cannot
allocate device memory.

The regular tridDmtsvStridedBatch allocates scratch for systems longer than
one warp holds; callers that reserve and account for all device memory up
front, or that run where an allocation's latency or failure is not
acceptable, use this variant instead: it keeps that scratch in one fixed
16 MiB device array inside the library. This file checks, through the C ABI,
that it gives the regular entry point's results (within the FP64 parity
tolerance of the other GPU tests) on several calls in a row, which share and
reuse the fixed array, that a problem needing more scratch than the
array holds is refused before anything runs, that a long-path call leaves
the device's free memory unchanged, and that zero pivots are reported
through the pivot word kept in the fixed array.

The file is named so that pytest collects it last; it passes run alone in a
fresh process (the first call sets up the array's device address) as well as
after the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from helpers import make_system, normwise
from tridsolver_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 normwise tolerance used by the GPU parity tests


def _no_alloc_entry():
    fn = _lib.load().tridDmtsvStridedBatchNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]
    return fn


def _ints(vals):
    return (ctypes.c_int * len(vals))(*vals)


def _solve_both(dims, solvedim, seed):
    a, b, c, d = make_system(dims, solvedim, np.float64, seed=seed)
    ta, tb_, tc = (torch.from_numpy(v).cuda() for v in (a, b, c))
    d_regular = torch.from_numpy(d).cuda()
    d_fixed = d_regular.clone()
    st_regular = tb.tridDmtsvStridedBatch(None, ta, tb_, tc, d_regular, len(dims), solvedim, dims,
                                          dims)
    st_fixed = _no_alloc_entry()(None, ta.data_ptr(), tb_.data_ptr(), tc.data_ptr(),
                                 d_fixed.data_ptr(), len(dims), solvedim, _ints(dims), _ints(dims))
    torch.cuda.synchronize()
    return st_regular, st_fixed, d_regular.cpu().numpy(), d_fixed.cpu().numpy()


# Long systems (the path that needs scratch), along x and along y, then a
# problem short enough to need none; the first case again at the end, after
# the array holds another call's leftovers.
CASES = [([100000], 0), ([3, 20000], 1), ([64, 48, 40], 1), ([30000, 5], 0), ([100000], 0)]


def test_calls_in_a_row_match_the_regular_entry_point():
    for seed, (dims, solvedim) in enumerate(CASES):
        st_regular, st_fixed, want, got = _solve_both(dims, solvedim, seed % 4)
        assert st_regular == tb.TridStatus.SUCCESS
        assert st_fixed == tb.TridStatus.SUCCESS
        assert normwise(got, want) <= TOL, (dims, solvedim)


def test_problem_beyond_the_fixed_array_is_refused():
    dims = [100000, 64]  # 64 long systems: about 26 MB of reduced rows
    arrs = [torch.ones(dims[0] * dims[1], dtype=torch.float64, device="cuda") for _ in range(4)]
    before = arrs[3].clone()
    st = _no_alloc_entry()(None, *(t.data_ptr() for t in arrs), 2, 0, _ints(dims), _ints(dims))
    torch.cuda.synchronize()
    assert st == tb.TridStatus.INVALID_VALUE
    assert torch.equal(arrs[3], before), "a refused call must not touch d"


def _call_fixed(arrs, dims, solvedim):
    return _no_alloc_entry()(None, *(t.data_ptr() for t in arrs), len(dims), solvedim, _ints(dims),
                             _ints(dims))


def test_long_path_takes_no_device_memory():
    """The property the entry point exists for: a long-path call (16 systems
    of 100000 rows, about 7 MB of reduced rows) leaves the device's free
    memory where it was, while the regular entry point takes its scratch
    from the library's pool, which keeps it until released."""
    dims = [100000, 16]
    a, b, c, d = make_system(dims, 0, np.float64, seed=7)
    arrs = [torch.from_numpy(v).cuda() for v in (a, b, c, d)]
    tb.release_scratch()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _call_fixed(arrs, dims, 0) == tb.TridStatus.SUCCESS
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 < (2 << 20), free0 - free1
    st = tb.tridDmtsvStridedBatch(None, *arrs, 2, 0, dims, dims)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    tb.release_scratch()
    assert st == tb.TridStatus.SUCCESS
    assert free1 - free2 >= (4 << 20), "the measurement sees the regular entry's scratch"


@pytest.mark.parametrize("dims", [[16, 8], [100000]])
def test_zero_pivot_reported_through_the_fixed_array(dims):
    """A zero pivot is reported by a blocking call (the pivot word is the
    first word of the fixed array), and the next clean call succeeds."""
    a, b, c, d = make_system(dims, 0, np.float64, seed=3)
    a[:] = 0.0
    c[:] = 0.0
    b[37] = 0.0
    arrs = [torch.from_numpy(v).cuda() for v in (a, b, c, d)]
    assert _call_fixed(arrs, dims, 0) == tb.TridStatus.ZERO_PIVOT
    a, b, c, d = make_system(dims, 0, np.float64, seed=3)
    arrs = [torch.from_numpy(v).cuda() for v in (a, b, c, d)]
    assert _call_fixed(arrs, dims, 0) == tb.TridStatus.SUCCESS
