"""GPU: the ADI heat timestep (native kernels, CUDA graph, differentiable form).

* tridDADIStep / tridSADIStep against the oracle's ADI step
  (oracle_adi_step_*: the 7-point RHS of apps/adi/src/preproc.hpp:173-214 and
  the x, y, z-Inc solves of adi_cpu.cpp:209-270), over several steps with
  per-step lambdas;
* a CUDA graph of one timestep, replayed, equals eager steps exactly;
* the differentiable timestep (native forward, native adjoint) equals the
  native one; its gradients with respect to the field and lambda equal those
  of the same step written with torch ops over the differentiable solve
  (the reference formulation below), and a multi-step run's gradients with
  respect to the initial field and every lambda match central finite
  differences; checkpointing gives the same gradients.
"""

import numpy as np
import pytest
import torch

from helpers import normwise
from oracle.pyoracle import Restatement
from tridsolver_b200.adi import ADIHeat, adi_run, adi_step
from tridsolver_b200.autograd import trid_solve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


def _field(shape, dtype, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    u = torch.randn(shape, generator=g, device="cuda", dtype=dtype)
    u[0], u[-1] = 0, 0
    u[:, 0], u[:, -1] = 0, 0
    u[:, :, 0], u[:, :, -1] = 0, 0
    return u


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
@pytest.mark.parametrize("shape", [(16, 18, 20), (9, 33, 64), (40, 6, 7), (3, 5, 600),
                                   (70, 3, 2), (24, 300, 20), (300, 12, 16),
                                   # y and z systems of 65-512 rows over x extents of
                                   # whole 128-byte groups (every chunk shape of the
                                   # streaming solves, Inc included)
                                   (130, 40, 64), (12, 257, 192), (300, 70, 128)])
@pytest.mark.parametrize("alpha", [1.0, 0.5])
@pytest.mark.parametrize("arrays", [False, True], ids=["fused", "arrays"])
def test_native_step_against_oracle(shape, dtype, tol, alpha, arrays, oracle):
    u = _field(shape, dtype)
    lams = np.random.default_rng(0).uniform(0.1, 1.0, 5)
    sim = ADIHeat(u.clone(), lams, alpha=alpha, coefficient_arrays=arrays)
    ref = u.cpu().numpy().reshape(-1).copy()
    nz, ny, nx = shape
    for k in range(5):
        sim.step()
        oracle.adi_step(ref, lams[k], -alpha * lams[k], 1 + 2 * alpha * lams[k], nx, ny, nz)
    torch.cuda.synchronize()
    assert int(sim.step_counter.item()) == 5
    assert normwise(sim.u.cpu().numpy().reshape(-1), ref) <= tol


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("shape", [(130, 200, 160), (72, 100, 300), (72, 300, 256)])
def test_fused_equals_arrays(shape, dtype):
    """Where both forms pick the same chunking (x: 129..512 rows, y and z:
    65..512 rows) the fused timestep runs the array timestep's right-hand-side
    arithmetic on coefficients factored once; the two agree to rounding
    (instruction selection, i.e. which products fuse into multiply-adds,
    differs between the kernels)."""
    u = _field(shape, dtype, seed=7)
    lams = np.random.default_rng(3).uniform(0.1, 1.0, 3)
    fused = ADIHeat(u.clone(), lams)
    arr = ADIHeat(u.clone(), lams, coefficient_arrays=True)
    fused.run(3)
    arr.run(3)
    torch.cuda.synchronize()
    tol = 1e-14 if dtype == torch.float64 else 1e-6
    assert normwise(fused.u.cpu().numpy(), arr.u.cpu().numpy()) <= tol
    assert normwise(fused.du.cpu().numpy(), arr.du.cpu().numpy()) <= tol


def test_graph_replay_equals_eager():
    u = _field((24, 20, 32), torch.float64, seed=3)
    lams = np.random.default_rng(1).uniform(0.1, 1.0, 12)
    eager = ADIHeat(u.clone(), lams)
    eager.run(11)
    graphed = ADIHeat(u.clone(), lams)
    graphed.capture()  # one eager warm-up step
    graphed.run(10)
    torch.cuda.synchronize()
    assert int(graphed.step_counter.item()) == 11
    assert torch.equal(eager.u, graphed.u)


def _torch_step(u, lam, alpha=1.0):
    """The timestep with torch ops and the differentiable solve: the
    reference formulation for the native adjoint (stencil, coefficient
    arrays with identity boundary rows, x, y, z solves)."""
    m = torch.zeros_like(u)
    m[1:-1, 1:-1, 1:-1] = 1
    a = -alpha * lam * m
    b = 1 + 2 * alpha * lam * m
    lap = torch.zeros_like(u)
    lap[1:-1, 1:-1, 1:-1] = (u[:-2, 1:-1, 1:-1] + u[2:, 1:-1, 1:-1] + u[1:-1, :-2, 1:-1] +
                             u[1:-1, 2:, 1:-1] + u[1:-1, 1:-1, :-2] + u[1:-1, 1:-1, 2:] -
                             6 * u[1:-1, 1:-1, 1:-1])
    du = lam * lap
    du = trid_solve(a, b, a, du, dim=2)
    du = trid_solve(a, b, a, du, dim=1)
    return u + trid_solve(a, b, a, du, dim=0)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-5)])
@pytest.mark.parametrize("shape", [(12, 14, 16), (5, 40, 9), (33, 6, 70), (3, 3, 3), (2, 7, 5),
                                   (130, 4, 3), (20, 300, 17),
                                   # an edge over 512: the coefficient-array form
                                   (4, 3, 600)])
@pytest.mark.parametrize("alpha", [1.0, 0.5])
def test_native_adjoint_equals_torch_formulation(shape, dtype, tol, alpha):
    u = torch.randn(shape, dtype=dtype, device="cuda")
    w = torch.randn(shape, dtype=dtype, device="cuda")
    grads = []
    for step in (adi_step, _torch_step):
        uu = u.clone().requires_grad_(True)
        lam = torch.tensor(0.43, dtype=dtype, device="cuda", requires_grad=True)
        (w * step(uu, lam, alpha)).sum().backward()
        grads.append((uu.grad.cpu().numpy(), lam.grad.item()))
    assert normwise(grads[0][0], grads[1][0]) <= tol
    assert abs(grads[0][1] - grads[1][1]) <= tol * max(1.0, abs(grads[1][1])) * 10


def test_torch_step_equals_native():
    u = _field((12, 14, 16), torch.float64, seed=4)
    lam = 0.37
    sim = ADIHeat(u.clone(), [lam])
    sim.step()
    out = adi_step(u, torch.tensor(lam, dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    assert normwise(out.cpu().numpy(), sim.u.cpu().numpy()) <= 1e-13


def test_backprop_through_steps_against_fd():
    shape = (8, 9, 10)
    u0 = _field(shape, torch.float64, seed=5)
    lams = torch.tensor(np.random.default_rng(2).uniform(0.1, 1.0, 6), dtype=torch.float64,
                        device="cuda")
    w = torch.randn(shape, dtype=torch.float64, device="cuda")

    def loss(u, lv, ck):
        return (w * adi_run(u, lv, checkpoint_every=ck)).sum()

    u_req = u0.clone().requires_grad_(True)
    l_req = lams.clone().requires_grad_(True)
    loss(u_req, l_req, 2).backward()
    gu, gl = u_req.grad.clone(), l_req.grad.clone()
    u2 = u0.clone().requires_grad_(True)
    l2 = lams.clone().requires_grad_(True)
    loss(u2, l2, 0).backward()
    assert torch.allclose(gu, u2.grad, rtol=1e-12, atol=1e-14)
    assert torch.allclose(gl, l2.grad, rtol=1e-12, atol=1e-14)
    h = 1e-6
    with torch.no_grad():
        for k in range(lams.shape[0]):
            lp, lm = lams.clone(), lams.clone()
            lp[k] += h
            lm[k] -= h
            fd = (loss(u0, lp, 0) - loss(u0, lm, 0)).item() / (2 * h)
            assert abs(fd - gl[k].item()) <= 1e-6 * max(1.0, abs(fd))
        idx = [(3, 4, 5), (2, 2, 2), (5, 6, 7)]
        for (i, j, kk) in idx:
            up, um = u0.clone(), u0.clone()
            up[i, j, kk] += h
            um[i, j, kk] -= h
            fd = (loss(up, lams, 0) - loss(um, lams, 0)).item() / (2 * h)
            assert abs(fd - gu[i, j, kk].item()) <= 1e-6 * max(1.0, abs(fd))
