"""GPU: FP32 solves refined to FP64 accuracy.

tridDmtsvStridedBatchRefine takes an FP64-specified system (FP64 a, b, c,
d): its FP32 factorisation is of the rounded coefficients, its residual of
the FP64 ones. The answer to match is the reference CPU solver (the library
built from scalar/src/cpu/trid_cpu.cpp, or the restatement where it is not
built) on the original FP64 coefficients: normwise relative error <= 1e-12
at every diagonal-dominance margin from 1e-3 to 1, along x, y and z, with
at least one refinement pass taken.

tridDmtsvStridedBatchMixed (below) takes FP32-stored coefficients.

The system is the FP32-stored coefficients taken exactly, so the FP64 oracle
(oracle/trid_oracle.c, the reference's Thomas recurrence) on the promoted
coefficients is the exact answer to match: normwise relative error <= 1e-12,
as for the plain FP64 path, across diagonal-dominance margins from 1e-3 to 1
(the precision configuration's range) and along x, y and z. Both strategies
are checked: the FP32 solve with FP64 refinement (mode 1, and the automatic
choice where the direct solve does not apply) and the direct FP64 solve of
the FP32 values (the automatic choice for strided 64 < N <= 512, which
reports 0 refinement passes).
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from helpers import make_system, normwise
from oracle.pyoracle import Reference, Restatement

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


@pytest.fixture(scope="module")
def checker():
    """The reference's own CPU solver when built, else the restatement."""
    try:
        return Reference()
    except FileNotFoundError:
        return Restatement()


def _problem(dims, solvedim, margin, seed):
    rng = np.random.default_rng(seed)
    shape = tuple(reversed(dims))
    marg = 10.0 ** rng.uniform(np.log10(margin), 0.0, shape) if margin < 1 else np.ones(shape)
    a, b, c, d = make_system(dims, solvedim, np.float64, seed=seed, margin=marg.reshape(shape))
    a32, b32, c32 = (v.astype(np.float32) for v in (a, b, c))
    return a32, b32, c32, d


SHAPES = [([512, 4, 3], 0), ([256, 8, 2], 0), ([200, 7], 0), ([33, 3], 0), ([1], 0),
          ([16, 512, 2], 1), ([10, 300], 1), ([24, 3, 512], 2), ([40, 5, 256], 2), ([9, 2, 7], 2),
          # rows a plane (>= 64 KiB) apart: the wide kernel's promoted form,
          # full and partial 32-system groups
          ([32, 256, 300], 2), ([20, 512, 130], 2), ([48, 256, 512], 2)]


def _problem64(dims, solvedim, margin, seed):
    """FP64-specified system with margins b - |a| - |c| log-uniform in
    [margin, 1] (all 1 for margin 1)."""
    rng = np.random.default_rng(seed)
    shape = tuple(reversed(dims))
    marg = 10.0 ** rng.uniform(np.log10(margin), 0.0, shape) if margin < 1 else np.ones(shape)
    return make_system(dims, solvedim, np.float64, seed=seed, margin=marg.reshape(shape))


@pytest.mark.parametrize("margin", [1e-3, 1e-2, 1e-1, 1.0])
@pytest.mark.parametrize("dims,solvedim", SHAPES + [([512, 6], 0), ([130, 2], 0)])
def test_refine_matches_fp64_specified_system(dims, solvedim, margin, checker):
    a, b, c, d = _problem64(dims, solvedim, margin, seed=7 * sum(dims) + solvedim)
    want = d.copy()
    checker.strided_batch(a, b, c, want, dims, solvedim)
    ta, tb_, tc, td = (torch.from_numpy(v).cuda() for v in (a, b, c, d))
    st, iters, est = tb.tridDmtsvStridedBatchRefine(None, ta, tb_, tc, td, len(dims), solvedim,
                                                    dims, dims, max_iters=12, tol=1e-13)
    assert st == 0
    assert 2 <= iters <= 12
    assert 0.0 <= est <= 1e-13
    err = normwise(td.cpu().numpy(), want)
    assert err <= 1e-12, (err, iters, est)
    # inputs untouched
    assert torch.equal(ta.cpu(), torch.from_numpy(a)) and torch.equal(tc.cpu(), torch.from_numpy(c))


def test_fp32_values_are_a_different_system(checker):
    """Why the FP64-specified form exists: the FP32-stored solve is exact for
    the rounded coefficients, which at margin 1e-3 lie far from the FP64
    system's solution."""
    dims, solvedim = [512, 16], 0
    a, b, c, d = _problem64(dims, solvedim, 1e-3, seed=11)
    want = d.copy()
    checker.strided_batch(a, b, c, want, dims, solvedim)
    ta, tb_, tc = (torch.from_numpy(v.astype(np.float32)).cuda() for v in (a, b, c))
    td = torch.from_numpy(d).cuda()
    st, _, _ = tb.tridDmtsvStridedBatchMixed(None, ta, tb_, tc, td, 2, 0, dims, dims)
    assert st == 0
    assert normwise(td.cpu().numpy(), want) > 1e-9


def test_refine_arguments():
    a = torch.ones(600 * 2, dtype=torch.float64, device="cuda")
    st, it, est = tb.tridDmtsvStridedBatchRefine(None, a, a, a, a.clone(), 2, 0, [600, 2], [600, 2])
    assert st == tb.TridStatus.MATRIX_TYPE_NOT_SUPPORTED and (it, est) == (-1, -1.0)
    st, _, _ = tb.tridDmtsvStridedBatchRefine(None, a, a, a, a.clone(), 2, 0, [600, 2], [600, 2],
                                              max_iters=0)
    assert st == tb.TridStatus.INVALID_VALUE
    st, it, est = tb.tridDmtsvStridedBatchRefine(None, a, a, a, a, 2, 0, [0, 2], [0, 2])
    assert (st, it, est) == (0, 0, 0.0)


@pytest.mark.parametrize("mode", [0, 1], ids=["auto", "refine"])
@pytest.mark.parametrize("margin", [1e-3, 1e-1, 1.0])
@pytest.mark.parametrize("dims,solvedim", SHAPES)
def test_mixed_matches_fp64_oracle(dims, solvedim, margin, mode, oracle):
    a32, b32, c32, d = _problem(dims, solvedim, margin, seed=sum(dims) + solvedim)
    want = d.copy()
    oracle.strided_batch(*(v.astype(np.float64) for v in (a32, b32, c32)), want, dims, solvedim)
    ta, tb_, tc = (torch.from_numpy(v).cuda() for v in (a32, b32, c32))
    td = torch.from_numpy(d).cuda()
    tb.set_mixed_mode(mode)
    try:
        st, iters, corr = tb.tridDmtsvStridedBatchMixed(None, ta, tb_, tc, td, len(dims), solvedim,
                                                        dims, dims, max_iters=12, tol=1e-13)
    finally:
        tb.set_mixed_mode(0)
    assert st == 0
    n = dims[solvedim]
    aligned_rows = solvedim == 0 and all(v % 4 == 0 for v in dims[:1])  # system starts 16-byte aligned
    direct = mode == 0 and ((solvedim >= 1 and 64 < n <= 512) or (aligned_rows and 128 < n <= 512))
    if direct:
        assert (iters, corr) == (0, 0.0)
    else:
        assert 1 <= iters <= 12
    err = normwise(td.cpu().numpy(), want)
    assert err <= 1e-12, (err, iters, corr)


def test_mixed_mode_argument():
    with pytest.raises(tb.TridError):
        tb.set_mixed_mode(3)
    tb.set_mixed_mode(2)
    tb.set_mixed_mode(0)


def test_mixed_unsupported_cases_are_reported():
    a32, b32, c32, d = _problem([600, 2], 0, 1.0, seed=1)
    ta, tb_, tc = (torch.from_numpy(v).cuda() for v in (a32, b32, c32))
    td = torch.from_numpy(d).cuda()
    st, _, _ = tb.tridDmtsvStridedBatchMixed(None, ta, tb_, tc, td, 2, 0, [600, 2], [600, 2])
    assert st == tb.TridStatus.MATRIX_TYPE_NOT_SUPPORTED
    st, _, _ = tb.tridDmtsvStridedBatchMixed(None, ta, tb_, tc, td, 2, 0, [600, 2], [600, 2],
                                             max_iters=0)
    assert st == tb.TridStatus.INVALID_VALUE
