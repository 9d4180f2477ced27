"""GPU: the generic strided surface (tridDsolveBatchedTrid / tridSsolveBatchedTrid
and Inc), the reference's solveBatchedTrid addressing
(scalar/src/cuda/trid_thomaspcr.hpp:794-832): the 3D cube examples of its
comment block (x, y with sub-batches, z), a partial last sub-batch, strides
the reference does not accept, separate d and x, and x += solution.

Each system is gathered into a contiguous array and solved by the oracle's
per-system Thomas recurrence (the reference's trid_scalar), then compared
normwise: <= 1e-12 (FP64), <= 1e-5 (FP32).
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


def _starts(num, stride1, stride2, sbs, sbstride):
    k = np.arange(num, dtype=np.int64)
    if stride1 == 1:
        return k * stride2
    return (k // sbs) * sbstride + (k % sbs) * stride2


def _case(num, length, stride1, stride2, sbs, sbstride, dt, inc, oracle, seed):
    starts = _starts(num, stride1, stride2, sbs, sbstride)
    idx = starts[:, None] + np.arange(length, dtype=np.int64)[None, :] * stride1
    size = int(idx.max()) + 1
    assert len(np.unique(idx)) == idx.size  # systems do not overlap
    rng = np.random.default_rng(seed)
    a = rng.uniform(-0.5, 0.5, size)
    c = rng.uniform(-0.5, 0.5, size)
    b = 1 + np.abs(a) + np.abs(c) + rng.uniform(0, 1, size)
    d = rng.standard_normal(size)
    x0 = rng.standard_normal(size) if inc else np.full(size, 7.0)
    a, b, c, d, x0 = (v.astype(dt) for v in (a, b, c, d, x0))
    # oracle: gather each system, per-system Thomas, scatter
    flat = idx.reshape(-1)
    ga, gb, gc, gd = (v[flat].astype(np.float64) for v in (a, b, c, d))
    offs = np.arange(num + 1, dtype=np.int64) * length
    oracle.ragged(ga, gb, gc, gd, offs)
    want = x0.astype(np.float64).copy()
    if inc:
        want[flat] += gd
    else:
        want[flat] = gd
    ta, tb_, tc, td, tx = (torch.from_numpy(v).cuda() for v in (a, b, c, d, x0))
    st = tb.solve_batched_trid(num, length, stride1, stride2, sbs, sbstride, ta, tb_, tc, td, tx,
                               inc=inc)
    assert st == 0
    got = tx.cpu().numpy().astype(np.float64)
    assert np.array_equal(td.cpu().numpy(), d)  # d is only read
    untouched = np.setdiff1d(np.arange(size), flat)
    assert np.array_equal(got[untouched], want[untouched])
    err = np.max(np.abs(got[flat] - want[flat])) / np.max(np.abs(want[flat]))
    return err


X, Y, Z = 40, 36, 30
CUBE = [  # the reference's examples for an X*Y*Z cube
    ("x", Y * Z, X, 1, X, Y * Z, 0),
    ("y", X * Z, Y, X, 1, X, X * Y),
    ("z", X * Y, Z, X * Y, 1, X * Y, 0),
]


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("name,num,length,s1,s2,sbs,sbst", CUBE)
def test_cube_examples(name, num, length, s1, s2, sbs, sbst, inc, dt, tol, oracle):
    assert _case(num, length, s1, s2, sbs, sbst, dt, inc, oracle, seed=len(name)) <= tol


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
@pytest.mark.parametrize("num,length,s1,s2,sbs,sbst", [
    (50, 300, 7, 1, 7, 7 * 300),       # partial last sub-batch (50 = 7*7 + 1)
    (64, 513, 3, 1, 3, 3 * 513),       # long systems, strided
    (33, 1000, 1, 1003, 1, 0),         # long contiguous systems, padded starts
    (20, 200, 5, 2, 2, 1000 * 5),      # stride1 and stride2 both != 1
    (12, 9, 1, 11, 1, 0),              # short systems (pure PCR)
])
def test_general_strides(num, length, s1, s2, sbs, sbst, dt, tol, oracle):
    assert _case(num, length, s1, s2, sbs, sbst, dt, False, oracle, seed=num + length) <= tol


def test_invalid_arguments():
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    assert tb.solve_batched_trid(-1, 4, 1, 4, 1, 0, t, t, t, t, t) == tb.TridStatus.INVALID_VALUE
    assert tb.solve_batched_trid(2, 4, 0, 4, 1, 0, t, t, t, t, t) == tb.TridStatus.INVALID_VALUE
    assert tb.solve_batched_trid(2, 4, 2, 1, 0, 8, t, t, t, t, t) == tb.TridStatus.INVALID_VALUE
    assert tb.solve_batched_trid(0, 4, 1, 4, 1, 0, t, t, t, t, t) == 0
