"""The merge loss as a torch.autograd.Function over the eight merge
parameters (test harness only; the product is the C ABI).

MergeLoss.apply(theta, setup) returns sum(weight * (merge(theta) - target)^2)
for the burst in `setup`; forward and gradient come from one call of
isa_merge_backward (Merger.backward: the forward merge, then the adjoint
kernels), so backward only scales the stored gradient by the upstream one.
theta holds (k_detail, k_denoise, dth, dtr, k_stretch, k_shrink, robust_s,
robust_t)."""
import numpy as np
import torch

from imagestackalignator_b200 import params as P

NAMES = ["k_detail", "k_denoise", "dth", "dtr", "k_stretch", "k_shrink", "robust_s", "robust_t"]


class MergeSetup:
    """What the loss is taken over: the burst (raw device frames, raw info, size),
    the other merge parameters, the target image and the per-pixel weight, and
    the Merger class to build a context with."""

    def __init__(self, merger_cls, width, height, frames, base_params, raw, info, target, weight):
        self.merger_cls = merger_cls
        self.width, self.height, self.frames = width, height, frames
        self.base = base_params
        self.raw, self.info, self.target, self.weight = raw, info, target, weight
        self.calls = 0

    def params(self, theta):
        p = P.MergeParams(**vars(self.base))
        for n, v in zip(NAMES, theta):
            setattr(p, n, float(v))
        return p


class MergeLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, setup):
        m = setup.merger_cls(setup.width, setup.height, setup.frames, setup.params(theta.detach().cpu().numpy()))
        try:
            _, loss, grad = m.backward(setup.raw, setup.info, setup.target, weight=setup.weight)
        finally:
            m.close()
        setup.calls += 1
        ctx.save_for_backward(torch.as_tensor(np.asarray(grad, np.float64), dtype=theta.dtype, device=theta.device))
        return theta.new_tensor(loss)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None
