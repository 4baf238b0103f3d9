"""Differentiable RBF-PUM transfer for PyTorch.

``rbf_pum_transfer(source_points, source_values, target_points, rbf_function)``
returns the transferred values and back-propagates to ``source_values``
(the transpose transfer) and to ``target_points`` (the gradient of the
partition-of-unity interpolant at the targets, with the patch membership
held fixed: membership changes are measure-zero events and are not
differentiated).  Both gradients come from the library's adjoint kernels
(pacman_b200_plan_adjoint); no gradient flows to ``source_points``.
"""
from __future__ import annotations

import torch

from .rbf import Plan


class _Transfer(torch.autograd.Function):
    @staticmethod
    def forward(ctx, source_values, target_points, source_points, rbf_function, opts):
        plan = Plan(source_points.shape[1], source_points.detach(), target_points.detach(),
                    **opts)
        out = plan.execute(rbf_function, source_values.detach(), save_for_adjoint=True)
        ctx.plan = plan
        if not torch.is_tensor(out):
            out = torch.from_numpy(out)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        need_v, need_t = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gv = gt = None
        if need_v or need_t:
            gv, gt = ctx.plan.adjoint(grad_out.detach().to(torch.float64).contiguous(),
                                      values=need_v, targets=need_t)
            if gv is not None and not torch.is_tensor(gv):
                gv = torch.from_numpy(gv)
            if gt is not None and not torch.is_tensor(gt):
                gt = torch.from_numpy(gt)
        return gv, gt, None, None, None


def rbf_pum_transfer(source_points, source_values, target_points, rbf_function, *,
                     nodes_per_cluster=50, relative_overlap=0.15, support_radius=0.1,
                     precision="fp64"):
    """Transfer with gradients to source_values and target_points."""
    opts = dict(nodes_per_cluster=nodes_per_cluster, relative_overlap=relative_overlap,
                support_radius=support_radius, precision=precision)
    return _Transfer.apply(source_values, target_points, source_points, rbf_function, opts)
