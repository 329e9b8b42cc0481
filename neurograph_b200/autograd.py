"""torch.autograd bridge: characteristic path length and global efficiency as differentiable functions of arc weights.

forward runs ngx_apsp_grad (the batched kernel computes the APSP summaries and, in the same launch, the adjoint of
both metrics with respect to every arc length); backward returns grad_cpl * dCPL/dw + grad_eff * dE/dw. Arc length is
|w| (AllPairsShortestPath.h via DijkstraCommon.h:36-54), so for positive weights d/dw = d/dlength; weights must be
positive here. The graph is rebuilt from the host CSR on every call, which suits tests and small optimisation loops.
"""

from __future__ import annotations

import numpy as np
import torch

from . import Graph


class ApspMetrics(torch.autograd.Function):
    """(w, n, row_ptr, col, sources) -> tensor([CPL, efficiency]) (float64); differentiable in w only."""

    @staticmethod
    def forward(ctx, w: torch.Tensor, n: int, row_ptr, col, sources=None):
        weights = w.detach().to("cpu", torch.float64).numpy()
        if weights.size and not (weights > 0).all():
            raise ValueError("ApspMetrics needs positive weights (length = |w|)")
        with Graph(n, np.asarray(row_ptr), np.asarray(col), weights) as g:
            dcpl, deff, r = g.apsp_grad(sources=sources)
        ctx.save_for_backward(torch.from_numpy(dcpl.copy()), torch.from_numpy(deff.copy()))
        ctx.w_device, ctx.w_dtype = w.device, w.dtype
        return torch.tensor([r.cpl, r.efficiency], dtype=torch.float64, device=w.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        dcpl, deff = ctx.saved_tensors
        g = grad_out.detach().to("cpu", torch.float64)
        grad_w = (g[0] * dcpl + g[1] * deff).to(ctx.w_device, ctx.w_dtype)
        return grad_w, None, None, None, None


def apsp_metrics(w: torch.Tensor, n: int, row_ptr, col, sources=None) -> torch.Tensor:
    """tensor([CPL, efficiency]) of the graph with arc weights w; backpropagates into w."""
    return ApspMetrics.apply(w, n, row_ptr, col, sources)
