"""GPU: the adjoint kernel and the autograd wrapper.

* against the oracle's transposed solve (oracle/trid_oracle.c
  oracle_adjoint_d: the reference's Thomas recurrence on T^T, then the
  products), normwise <= 1e-12, along x, y and z, with and without the
  a/b/c gradients;
* against FP64 central finite differences (h = 1e-6) of L = sum(w * x) on
  random entries of a, b, c and d;
* torch.autograd.gradcheck of the wrapper on a small FP64 problem.
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from helpers import make_system, normwise
from oracle.pyoracle import Restatement
from tridsolver_b200.autograd import trid_solve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


SHAPES = [([64, 12, 5], 0), ([9, 40, 6], 1), ([7, 5, 33], 2), ([512, 3], 0), ([6, 700], 1),
          ([1, 1, 1], 2), ([2, 2], 1), ([16, 256, 4], 1),
          # the streaming kernel's adjoint form (strided, 64 < N <= 512): every
          # chunk size, partial groups and chunks, y and z layouts
          ([32, 100, 3], 1), ([20, 5, 300], 2), ([48, 2, 512], 2), ([16, 129, 2], 1)]


@pytest.mark.parametrize("products", [True, False])
@pytest.mark.parametrize("dims,solvedim", SHAPES)
def test_adjoint_against_oracle(dims, solvedim, products, oracle):
    a, b, c, d = make_system(dims, solvedim, np.float64, seed=sum(dims))
    x = d.copy()
    oracle.strided_batch(a, b, c, x, dims, solvedim)
    w = np.random.default_rng(1).standard_normal(d.size)
    want = oracle.adjoint(a, b, c, x, w, dims, solvedim)
    ta, tb_, tc, tx, tw = (torch.from_numpy(v).cuda() for v in (a, b, c, x, w))
    outs = [torch.full_like(tx, np.nan) for _ in range(4)]
    abar, bbar, cbar, dbar = outs if products else (None, None, None, outs[3])
    st = tb.tridDmtsvStridedBatchAdjoint(None, ta, tb_, tc, tx, tw, dbar, abar, bbar, cbar,
                                         len(dims), solvedim, dims, dims)
    torch.cuda.synchronize()
    assert st == 0
    assert normwise(outs[3].cpu().numpy(), want[3]) <= 1e-12
    if products:
        for got, ref in zip(outs[:3], want[:3]):
            assert normwise(got.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("which", [(True, False, False), (False, True, True), (False, False, True)])
def test_adjoint_some_products(which, oracle):
    """Only some of abar, bbar, cbar asked for (the others null), on the
    streaming path: the ones asked for match the oracle, dbar too."""
    dims, sd = [24, 7, 260], 2
    a, b, c, d = make_system(dims, sd, np.float64, seed=8)
    x = d.copy()
    oracle.strided_batch(a, b, c, x, dims, sd)
    w = np.random.default_rng(2).standard_normal(d.size)
    want = oracle.adjoint(a, b, c, x, w, dims, sd)
    ta, tb_, tc, tx, tw = (torch.from_numpy(v).cuda() for v in (a, b, c, x, w))
    outs = [torch.full_like(tx, np.nan) if k < 3 and which[k] else None for k in range(3)]
    dbar = torch.full_like(tx, np.nan)
    st = tb.tridDmtsvStridedBatchAdjoint(None, ta, tb_, tc, tx, tw, dbar, outs[0], outs[1], outs[2],
                                         3, sd, dims, dims)
    torch.cuda.synchronize()
    assert st == 0
    assert normwise(dbar.cpu().numpy(), want[3]) <= 1e-12
    for k in range(3):
        if which[k]:
            assert normwise(outs[k].cpu().numpy(), want[k]) <= 1e-12


@pytest.mark.parametrize("dims,sd", [([20, 30, 4], 1), ([40, 3, 200], 2)])
def test_adjoint_fp32(dims, sd, oracle):
    a, b, c, d = make_system(dims, sd, np.float64, seed=3)
    x = d.copy()
    oracle.strided_batch(a, b, c, x, dims, sd)
    w = np.random.default_rng(1).standard_normal(d.size)
    want = oracle.adjoint(a, b, c, x, w, dims, sd)
    t = [torch.from_numpy(v.astype(np.float32)).cuda() for v in (a, b, c, x, w)]
    outs = [torch.empty_like(t[0]) for _ in range(4)]
    st = tb.tridSmtsvStridedBatchAdjoint(None, *t, outs[3], outs[0], outs[1], outs[2], 3, sd, dims,
                                         dims)
    torch.cuda.synchronize()
    assert st == 0
    for got, ref in zip(outs, want):
        assert normwise(got.cpu().numpy(), ref) <= 1e-5


def test_autograd_against_finite_differences(oracle):
    dims, sd = [6, 24, 5], 1
    a, b, c, d = make_system(dims, sd, np.float64, seed=7)
    w = np.random.default_rng(2).standard_normal(d.size)
    ts = [torch.from_numpy(v).cuda().reshape(tuple(reversed(dims))).requires_grad_(True)
          for v in (a, b, c, d)]
    tw = torch.from_numpy(w).cuda().reshape(tuple(reversed(dims)))
    x = trid_solve(*ts, dim=2 - sd)
    (x * tw).sum().backward()
    grads = [t.grad.reshape(-1).cpu().numpy() for t in ts]

    def loss(arrs):
        xx = arrs[3].copy()
        oracle.strided_batch(arrs[0], arrs[1], arrs[2], xx, dims, sd)
        return float(np.dot(w, xx))

    rng = np.random.default_rng(5)
    h = 1e-6
    for k in range(4):
        for idx in rng.integers(0, d.size, 25):
            p = [v.copy() for v in (a, b, c, d)]
            m = [v.copy() for v in (a, b, c, d)]
            p[k][idx] += h
            m[k][idx] -= h
            fd = (loss(p) - loss(m)) / (2 * h)
            assert abs(fd - grads[k][idx]) <= 1e-6 * max(1.0, abs(fd)), (k, idx, fd, grads[k][idx])


def test_gradcheck():
    g = torch.Generator(device="cuda").manual_seed(0)
    shape = (3, 4, 6)
    a = (torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) - 0.5)
    c = (torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) - 0.5)
    b = 1.5 + a.abs() + c.abs()
    d = torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
    for dim in range(3):
        args = [t.clone().requires_grad_(True) for t in (a, b, c, d)]
        assert torch.autograd.gradcheck(lambda *t: trid_solve(*t, dim=dim), args, eps=1e-6,
                                        atol=1e-8, rtol=1e-6)
