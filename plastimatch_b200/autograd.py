"""Optional PyTorch binding of the cost function, for checks.

``bspline_score(coeff, ctx, ...)`` is a ``torch.autograd.Function``: the
forward pass is one ``bspline_score()`` evaluation through the C ABI
(``b200bsp_score``: similarity metric times lambda plus the analytic
regulariser) and the backward pass returns the library's analytic gradient
-- the hand-written adjoint kernels' output -- scaled by the incoming
gradient.  Nothing is differentiated by autograd through the kernels; the
binding only lets torch tools (``torch.autograd.grad``, ``gradcheck``-style
finite differences, optimisers) drive the product's own gradient path.

The score is a float32 scalar as the reference's ``Bspline_score`` keeps it;
``coeff`` may live on the CPU or on a GPU (it is copied to the host for the
call; the gradient comes back on ``coeff``'s device and dtype).
"""
from __future__ import annotations

import numpy as np
import torch

from . import Context, RegParms

__all__ = ["bspline_score"]


class _BsplineScore(torch.autograd.Function):
    @staticmethod
    def forward(fctx, coeff, ctx, metric, lam, reg):
        c = np.ascontiguousarray(
            coeff.detach().to("cpu", torch.float32).numpy())
        total, grad, _smetric, _nvox = ctx.score(c, metric=metric, lam=lam,
                                                 reg=reg)
        fctx.save_for_backward(
            torch.from_numpy(grad).to(device=coeff.device, dtype=coeff.dtype))
        return torch.tensor(total, dtype=torch.float32, device=coeff.device)

    @staticmethod
    def backward(fctx, grad_out):
        (g,) = fctx.saved_tensors
        return grad_out.to(g.dtype) * g, None, None, None, None


def bspline_score(coeff: torch.Tensor, ctx: Context, metric: str = "mse",
                  lam: float = 1.0, reg: RegParms | None = None
                  ) -> torch.Tensor:
    """Total score of ``bspline_score()`` at ``coeff`` (num_coeff floats,
    xyz interleaved per knot), differentiable with respect to ``coeff``
    through the analytic gradient."""
    if coeff.dim() != 1 or coeff.numel() != ctx.num_coeff:
        raise ValueError(f"coeff must hold {ctx.num_coeff} values")
    return _BsplineScore.apply(coeff, ctx, metric, lam, reg)
