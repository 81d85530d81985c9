"""Differentiable FMM matvec: a torch.autograd.Function whose backward is the
hand-written adjoint FMM (``pbbfmm_compute_adjoint_device``).

    out = fmm_matvec(tree, target, source, weight)          # (nCols, Nf)
    loss = (out * g).sum(); loss.backward()
    weight.grad  == K^T g                 (the transposed pass on the same tree)
    source.grad  == sum_c w_c grad_y phi_c  (differentiated interpolation + kernel gradient)
    target.grad  == sum_c g_c grad_x f_c

Shapes: target (Nf, 3), source (Ns, 3), weight (nCols, Ns) -- float64 CUDA
tensors.  The forward pass accumulates nothing: out is a fresh tensor.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import H2_3D_Tree, compute_adjoint_device, compute_device


class FMMMatvec(torch.autograd.Function):
    @staticmethod
    def forward(ctx, target, source, weight, tree, precision):
        target = target.contiguous()
        source = source.contiguous()
        weight = weight.contiguous()
        nCols = weight.shape[0]
        out = torch.zeros(nCols, target.shape[0], dtype=torch.float64, device=target.device)
        compute_device(tree, target, source, weight, nCols, out, precision=precision)
        ctx.save_for_backward(target, source, weight)
        ctx.tree = tree
        ctx.precision = precision
        return out

    @staticmethod
    def backward(ctx, g):
        target, source, weight = ctx.saved_tensors
        g = g.contiguous()
        nCols = weight.shape[0]
        need_t, need_s, need_w = ctx.needs_input_grad[:3]
        gw = torch.zeros_like(weight) if need_w else None
        gs = torch.zeros_like(source) if need_s else None
        gt = torch.zeros_like(target) if need_t else None
        if need_t or need_s or need_w:
            compute_adjoint_device(ctx.tree, target, source, weight, g, nCols, grad_weight=gw,
                                   grad_source=gs, grad_target=gt, precision=ctx.precision)
        return gt, gs, gw, None, None


def fmm_matvec(tree: H2_3D_Tree, target: torch.Tensor, source: torch.Tensor,
               weight: torch.Tensor, precision: Optional[int] = None) -> torch.Tensor:
    """K(target, source) @ weight^T as (nCols, Nf), differentiable in all three."""
    prec = tree.precision if precision is None else int(precision)
    return FMMMatvec.apply(target, source, weight, tree, prec)
