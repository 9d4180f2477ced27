"""GPU: the reference's own CUDA library, built for sm_100a, as a comparator.

bench.py times scalar/src/cuda/trid_cuda.cu (oracle/_ref/libtridcuda_ref.so,
compiled from the reference's sources by oracle/Makefile) beside this
library on the same B200. Before its numbers mean anything it must be doing
the same work: here its results, with its default opts, match the
restatement oracle (FP64 normwise 1e-12, FP32 1e-5) along x, y and z,
overwrite and Inc, on shapes its vectorised paths accept (x a multiple of 8),
and on the headline 256^3 grid against this library's own result.
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from helpers import make_system, normwise
from oracle.pyoracle import ReferenceGPU, Restatement

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-12, np.float32: 1e-5}


@pytest.fixture(scope="module")
def refgpu():
    try:
        return ReferenceGPU()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(f"reference CUDA library not built: {e}")


@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim", [([64, 48, 40], 0), ([64, 48, 40], 1), ([64, 48, 40], 2),
                                           ([128, 96], 0), ([128, 96], 1)])
def test_reference_gpu_matches_oracle(dims, solvedim, dt, inc, refgpu):
    a, b, c, d = make_system(dims, solvedim, dt, seed=31 + solvedim)
    u0 = np.random.default_rng(5).standard_normal(d.size).astype(dt) if inc else None
    want_d, want_u = d.copy(), (u0.copy() if inc else None)
    Restatement().strided_batch(a, b, c, want_d, dims, solvedim, u=want_u)
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in (a, b, c, d))
    tu = torch.from_numpy(u0).cuda() if inc else None
    refgpu.strided_batch(ta.data_ptr(), tb_.data_ptr(), tc.data_ptr(), td.data_ptr(), dims,
                         solvedim, ta.element_size(), u=tu.data_ptr() if inc else None)
    torch.cuda.synchronize()
    got = (tu if inc else td).cpu().numpy()
    assert normwise(got, want_u if inc else want_d) <= TOL[dt]


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_reference_gpu_matches_this_library_on_256_cubed(solvedim, refgpu):
    n = 256
    g = torch.Generator(device="cuda").manual_seed(solvedim)
    shape = (n, n, n)
    a = torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) - 0.5
    c = torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) - 0.5
    b = 1 + a.abs() + c.abs() + torch.rand(shape, generator=g, device="cuda", dtype=torch.float64)
    d = torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
    d2 = d.clone()
    refgpu.strided_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), d.data_ptr(), [n] * 3, solvedim, 8)
    assert tb.tridDmtsvStridedBatch(None, a, b, c, d2, 3, solvedim, [n] * 3, [n] * 3) == 0
    torch.cuda.synchronize()
    assert normwise(d.cpu().numpy(), d2.cpu().numpy()) <= 1e-12
