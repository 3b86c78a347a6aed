"""torch.autograd.Function over the off-grid objective (gs_score_grad).

A thin wrapper for gradient-check harnesses: forward evaluates the objective
and its gradient in one C-ABI call (the adjoint kernels), backward returns
the stored gradient scaled by the incoming one.  The parameters of each pick
are a row (angle, dx, dy, defocus, dfdiff, dfang) of a float tensor; the
pick's window, template and map position are fixed.
"""
from __future__ import annotations

import numpy as np
import torch

from . import REFINE_PICK_DTYPE, Context

PARAM_FIELDS = ("angle", "dx", "dy", "defocus", "dfdiff", "dfang")
GRAD_FIELDS = ("d_angle", "d_dx", "d_dy", "d_defocus", "d_dfdiff", "d_dfang")


class PickScore(torch.autograd.Function):
    """scores = PickScore.apply(params, ctx, base_picks); params: (n, 6)."""

    @staticmethod
    def forward(fctx, params: torch.Tensor, ctx: Context, base_picks: np.ndarray) -> torch.Tensor:
        pk = np.array(base_picks, dtype=REFINE_PICK_DTYPE, copy=True)
        p = params.detach().cpu().double().numpy()
        for k, f in enumerate(PARAM_FIELDS):
            pk[f] = p[:, k]
        res = ctx.score_grad(pk, with_gradient=True)
        g = np.stack([res[f].astype(np.float64) for f in GRAD_FIELDS], axis=1)
        fctx.save_for_backward(torch.from_numpy(g).to(params.dtype))
        return torch.from_numpy(res["score"].astype(np.float64)).to(params.dtype)

    @staticmethod
    def backward(fctx, grad_out: torch.Tensor):
        (g,) = fctx.saved_tensors
        return grad_out[:, None] * g, None, None
