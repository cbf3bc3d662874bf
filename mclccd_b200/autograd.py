"""torch.autograd.Function over the CCD forward and the toi adjoint.

``contact_toi(V0, V1, F, eta)`` runs update + traverse on CUDA tensors and
returns (toi, sten, is_vf) for the hits.  toi is the reference's ACCD value
(bit-identical), and it is differentiable in V0 and V1: the backward calls
``mclccd_tree_vjp_toi``, the adjoint of the contact time t* that toi
approximates (the first root of dist(x(t)) = eta at or after toi; hits that
never reach eta within the step, grazing hits and toi = 0 get zero gradient).
"""
from __future__ import annotations

import numpy as np
import torch

from .ccd import PREC_FP64, BVHTree


class _ContactToi(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V0, V1, F, eta, precision):
        tree = BVHTree(V0.shape[1], precision=precision)
        tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = float(eta)
        V0d, V1d = V0.detach().contiguous(), V1.detach().contiguous()
        tree.update(V0d, V1d, F.contiguous())
        tree.traverse()
        sten, is_vf, toi = tree.hits()
        ctx.tree = tree
        ctx.keep = (V0d, V1d)   # the adjoint reads the traverse's device arrays
        out_sten = torch.from_numpy(np.ascontiguousarray(sten)).to(V0.device)
        out_vf = torch.from_numpy(np.ascontiguousarray(is_vf)).to(V0.device)
        ctx.mark_non_differentiable(out_sten, out_vf)
        return torch.from_numpy(np.ascontiguousarray(toi)).to(V0.device), out_sten, out_vf

    @staticmethod
    def backward(ctx, g_toi, _g_sten, _g_vf):
        dV0, dV1, _ = ctx.tree.vjp_toi(g_toi.to(torch.float64).contiguous())
        return dV0, dV1, None, None, None


def contact_toi(V0: torch.Tensor, V1: torch.Tensor, F: torch.Tensor, eta: float, precision: int = PREC_FP64):
    """(toi, sten, is_vf) of the CCD hits between V0 and V1 (CUDA float64
    tensors, F int32 faces / edges); toi carries the contact-time gradient."""
    if not (V0.is_cuda and V1.is_cuda and F.is_cuda):
        raise ValueError("contact_toi takes CUDA tensors")
    return _ContactToi.apply(V0, V1, F, eta, precision)
