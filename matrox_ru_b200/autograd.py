"""torch.autograd.Function over the C-ABI: forward Y = K~ W, backward dL/dW = K~^T dL/dY.

K~ is not symmetric for H2-b (near lists are not symmetrised, ``sympiler/ClusterTree.cpp:556-573``
keeps that code commented out), so the gradient runs the hand-written transposed traversal
(every near block and far coupling transposed), not a second forward pass.
"""
from __future__ import annotations

import torch


class KernelMatVec(torch.autograd.Function):
    @staticmethod
    def forward(ctx, W, evaluator):
        ctx.evaluator = evaluator
        ctx.dtype = W.dtype
        Y = evaluator(W.detach().to(torch.float64).contiguous())
        return Y.to(W.dtype)

    @staticmethod
    def backward(ctx, G):
        GW = ctx.evaluator.adjoint(G.detach().to(torch.float64).contiguous())
        return GW.to(ctx.dtype), None
