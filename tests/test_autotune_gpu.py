"""GPU: the autotuner of strided and contiguous batches (tridAutotune).

For shapes of every layout class and length range, the tuned plan becomes
the automatic plan of its shape class (tridDescribePlan shows it), keeps
parity with the oracle (normwise 1e-12 FP64 / 1e-5 FP32, overwrite and
Inc), yields to tridForce* settings, and is forgotten by tridAutotuneReset.
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from helpers import make_system, normwise
from oracle.pyoracle import Restatement

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-12, np.float32: 1e-5}


@pytest.fixture(autouse=True)
def _reset():
    tb.autotune_reset()
    tb.force_plan()
    tb.force_stream(-1)
    yield
    tb.autotune_reset()
    tb.force_plan()
    tb.force_stream(-1)


SHAPES = [([20, 300], 0), ([256, 64, 16], 0), ([512, 40, 8], 0), ([3000, 6], 0),
          ([64, 256, 8], 1), ([40, 100, 6], 1), ([48, 512, 100], 2), ([33, 256, 300], 2),
          ([16, 16, 40], 2)]


@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim", SHAPES)
def test_tuned_plan_keeps_parity(dims, solvedim, dt, inc):
    es = np.dtype(dt).itemsize
    ms, plan = tb.autotune(es, dims, solvedim, inc=inc)
    assert ms > 0 and plan
    if not inc:
        assert tb.describe_plan(es, dims, solvedim) == plan
    a, b, c, d = make_system(dims, solvedim, dt, seed=sum(dims))
    u0 = np.random.default_rng(9).standard_normal(d.size).astype(dt) if inc else None
    want_d, want_u = d.copy(), (u0.copy() if inc else None)
    Restatement().strided_batch(a, b, c, want_d, dims, solvedim, u=want_u)
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in (a, b, c, d))
    if inc:
        tu = torch.from_numpy(u0).cuda()
        fn = tb.tridDmtsvStridedBatchInc if es == 8 else tb.tridSmtsvStridedBatchInc
        st = fn(None, ta, tb_, tc, td, tu, len(dims), solvedim, dims, dims)
        got = tu.cpu().numpy()
    else:
        fn = tb.tridDmtsvStridedBatch if es == 8 else tb.tridSmtsvStridedBatch
        st = fn(None, ta, tb_, tc, td, len(dims), solvedim, dims, dims)
        got = td.cpu().numpy()
    assert st == 0
    assert normwise(got, want_u if inc else want_d) <= TOL[dt]


def test_forced_settings_and_reset_take_precedence():
    dims, sd = [48, 512, 100], 2
    default = tb.describe_plan(8, dims, sd)
    _, tuned = tb.autotune(8, dims, sd)
    assert tb.describe_plan(8, dims, sd) == tuned
    # the same class (another length in the bucket, another count of systems)
    assert tb.describe_plan(8, [40, 512, 120], sd).split()[0] == tuned.split()[0]
    tb.force_stream(0)
    assert "stream" not in tb.describe_plan(8, dims, sd) and "wide" not in tb.describe_plan(8, dims, sd)
    tb.force_stream(-1)
    tb.autotune_reset()
    assert tb.describe_plan(8, dims, sd) == default
