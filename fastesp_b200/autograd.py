"""Differentiable ESP: ``esp(density, points, wfn, basis)`` as a torch autograd op.

Forward: the GPU pair-table build and evaluation (``build_table(...).esp``).
Backward: the hand-written adjoint kernels of the C ABI (``fe_esp_adjoint``):

* dL/dC  = dL/dV * dV/dC, the field kernel (a R^(a-e) F_m - 2p R R^a F_(m+1));
* dL/dP  = the point-weighted pair moments sum_i w_i R^a F_m carried back through
  the G contraction and the Hermite coefficients (recomputed per pair on the
  device, never stored) to the Cartesian density entries.

The screening decision of the build (which primitive pairs are kept) is held
fixed, so the gradient is that of the screened table.  The backward pass is
FP64 whatever precision the forward evaluation used.
"""
from __future__ import annotations

import torch

from .table import build_table


class _ESPFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, density, points, wfn, basis, tol, rule, precision):
        pts = points.detach().contiguous()
        table = build_table(wfn, basis, density.detach().contiguous(), pts, tol=tol, rule=rule)
        v = table.esp(pts, precision=precision)
        ctx.table = table
        ctx.save_for_backward(pts)
        return v

    @staticmethod
    def backward(ctx, grad_v):
        (pts,) = ctx.saved_tensors
        need_p, need_c = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        dP = dC = None
        if need_p or need_c:
            dP, dC = ctx.table.adjoint(pts, grad_v.detach().contiguous(),
                                       density=need_p, coords=need_c)
        return dP, dC, None, None, None, None, None


def esp(density, points, wfn, basis, tol: float = 1e-12, rule: str = "numpy",
        precision: str = "fp64"):
    """V(points) (n,) for the Cartesian ``density`` (n_func, n_func), both CUDA
    float64 tensors; differentiable with respect to both."""
    if not (torch.is_tensor(density) and torch.is_tensor(points)):
        raise TypeError("density and points must be torch tensors")
    return _ESPFunction.apply(density, points.reshape(-1, 3), wfn, basis, tol, rule, precision)
