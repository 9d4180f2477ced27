"""Differentiable batched tridiagonal solve for PyTorch.

``trid_solve(a, b, c, d, dim)`` returns x with T x = d along torch dimension
`dim` (a, b, c, d contiguous CUDA tensors of one shape and dtype). Forward
calls the library's strided solve; backward calls its adjoint kernel
(tridDmtsvStridedBatchAdjoint / tridSmtsvStridedBatchAdjoint), which solves
T^T dbar = dL/dx and forms dL/da, dL/db, dL/dc from the stored forward x in
one pass. Gradients of inputs that do not require them are not computed.
a[0] and c[N-1] along `dim` do not enter the solve and get zero gradient.

Both passes run on torch's current stream without blocking.
"""

import torch

from . import api


def _layout(t, dim):
    shape = tuple(t.shape)
    nd = len(shape)
    if not 1 <= nd <= api.MAXDIM:
        raise ValueError("1 to 3 dimensions")
    dims = list(reversed(shape))
    return dims, nd - 1 - (dim % nd)


class TridSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, b, c, d, dim):
        for t in (a, b, c, d):
            if t.shape != d.shape or not t.is_cuda or t.dtype != d.dtype:
                raise ValueError("a, b, c, d: CUDA tensors of one shape and dtype")
        a, b, c = (t.contiguous() for t in (a, b, c))
        x = d.contiguous().clone()
        dims, solvedim = _layout(x, dim)
        api.strided_batch(a, b, c, x, solvedim, dims)
        ctx.save_for_backward(a, b, c, x)
        ctx.dim = dim
        return x

    @staticmethod
    def backward(ctx, w):
        a, b, c, x = ctx.saved_tensors
        w = w.contiguous()
        dims, solvedim = _layout(x, ctx.dim)
        need_a, need_b, need_c, need_d = ctx.needs_input_grad[:4]
        dbar = torch.empty_like(x)
        abar = torch.empty_like(x) if need_a else None
        bbar = torch.empty_like(x) if need_b else None
        cbar = torch.empty_like(x) if need_c else None
        fn = (api.tridDmtsvStridedBatchAdjoint if x.dtype == torch.float64
              else api.tridSmtsvStridedBatchAdjoint)
        with torch.cuda.device(x.device), api.on_stream(blocking=False):
            st = fn(None, a, b, c, x, w, dbar, abar, bbar, cbar, len(dims), solvedim, dims, dims)
        if st != 0:
            raise api.TridError(st, "adjoint solve")
        return abar, bbar, cbar, (dbar if need_d else None), None


def trid_solve(a, b, c, d, dim=-1):
    """x = T^{-1} d along `dim`, differentiable in a, b, c and d."""
    return TridSolve.apply(a, b, c, d, dim)
