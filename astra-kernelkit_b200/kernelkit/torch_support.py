"""PyTorch autograd bridge (``kernelkit/torch_support.py`` of the
reference).

``AutogradOperator`` applies an operator to every (batch, channel) slice of
a 5D tensor; its backward applies ``op.T``, which for ``XrayTransform`` is
the reference's (scaled, unmatched) backprojector and for
``ExactXrayTransform`` the exact adjoint of the forward projector. Everything runs on the
current torch stream, so the modules can be captured in CUDA graphs.
"""
from __future__ import annotations

from itertools import product

import torch
from torch.autograd import Function

from .operator import BaseOperator, ExactXrayTransform, XrayTransform


class AutogradOperator(Function):
    """Autograd function for ``Operator`` objects (``torch_support.py:
    10-34``)."""

    @staticmethod
    def forward(ctx, input, op: BaseOperator):
        B, C = input.shape[:2]
        ctx.operator = op
        out = input.new_empty(B, C, *op.range_shape, dtype=torch.float32)
        x = input.detach()
        for s in product(range(B), range(C)):
            op(x[s], out=out[s])
        return out

    @staticmethod
    def backward(ctx, grad_output):
        op = ctx.operator
        B, C = grad_output.shape[:2]
        grad_input = grad_output.new_zeros(B, C, *op.domain_shape,
                                           dtype=torch.float32)
        g = grad_output.detach().contiguous()
        for s in product(range(B), range(C)):
            op.T(g[s], out=grad_input[s])
        return grad_input, None


class XrayForwardProjection(torch.nn.Module):
    """Module applying ``XrayTransform`` (``torch_support.py:37-45``)."""

    def __init__(self, *args, **kwargs):
        super().__init__()
        self.op = XrayTransform(*args, **kwargs)

    def forward(self, input):
        return AutogradOperator.apply(input, self.op)


class XrayBackprojection(torch.nn.Module):
    """Module applying ``XrayTransform.T`` (``torch_support.py:48-56``)."""

    def __init__(self, *args, **kwargs):
        super().__init__()
        self.op = XrayTransform(*args, **kwargs)

    def forward(self, input):
        return AutogradOperator.apply(input, self.op.T)


class ExactXrayForwardProjection(torch.nn.Module):
    """Forward projection whose backward pass is the exact adjoint of the
    ray-driven projector (``ExactXrayTransform``), so gradients of losses
    on ``A x`` are the true gradients: ``<A x, y> = <x, A^T y>`` to float32
    rounding. Arguments as ``ExactXrayTransform``. Angles are processed in
    chunks in the backward pass, recomputing the ray set-ups per chunk, so
    the extra memory stays bounded (``RayDrivenConeFP.adjoint_work_bytes``)
    for any volume size."""

    def __init__(self, *args, **kwargs):
        super().__init__()
        self.op = ExactXrayTransform(*args, **kwargs)

    def forward(self, input):
        return AutogradOperator.apply(input, self.op)


__all__ = ["AutogradOperator", "XrayForwardProjection", "XrayBackprojection",
           "ExactXrayForwardProjection"]
