"""Adam fit of the eight merge parameters through the adjoint of the merge
(isa_merge_backward), on one GPU or data-parallel over ranks.

The parameters (k_detail, k_denoise, dth, dtr, k_stretch, k_shrink,
robust_s, robust_t) are all positive and span four decades, so the fit runs
in log space from a starting point (the reference defaults): theta =
theta0 * exp(u), d loss / d u = theta * d loss / d theta. With a
torch.distributed process group, each rank merges its own bursts and the
loss and the eight gradients are summed over the ranks with one all-reduce
per step (NCCL between GPUs, gloo on CPU): every rank then takes the same
step and holds the same parameters, the data-parallel form of a fit over
many bursts. No counterpart in the reference, which has no gradients.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

NAMES = ("k_detail", "k_denoise", "dth", "dtr", "k_stretch", "k_shrink", "robust_s", "robust_t")


def adam_fit(grad_fn: Callable[[np.ndarray], Tuple[float, np.ndarray]], theta0: Sequence[float], steps: int, lr: float = 0.02,
             beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-12, group=None) -> Tuple[np.ndarray, List[float]]:
    """Adam in log space. grad_fn(theta) returns (loss, gradient) for this
    rank's share of the data; with a process group both are summed over the
    ranks before each step. Returns the final parameters and the loss of
    every step (summed over the ranks)."""
    theta0 = np.asarray(theta0, np.float64)
    u = np.zeros_like(theta0)
    m = np.zeros_like(theta0)
    v = np.zeros_like(theta0)
    losses = []
    for step in range(1, steps + 1):
        theta = theta0 * np.exp(u)
        loss, g = grad_fn(theta)
        g = np.asarray(g, np.float64)
        if group is not None:
            loss, g = _all_reduce(loss, g, group)
        losses.append(float(loss))
        gu = g * theta
        m = beta1 * m + (1 - beta1) * gu
        v = beta2 * v + (1 - beta2) * gu * gu
        u = u - lr * (m / (1 - beta1 ** step)) / (np.sqrt(v / (1 - beta2 ** step)) + eps)
    return theta0 * np.exp(u), losses


def _all_reduce(loss: float, g: np.ndarray, group) -> Tuple[float, np.ndarray]:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(np.concatenate([[loss], g]), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    return float(t[0]), t[1:]


def merger_grad_fn(merger, base_params, raw, info, target, weight=None, out=None):
    """grad_fn for adam_fit over one burst on one Merger: each call sets the
    eight parameters on the context (isa_ctx_set_params) and runs the forward
    merge and its adjoint (isa_merge_backward) against `target`."""
    from . import params as P

    def fn(theta):
        q = P.MergeParams(**vars(base_params))
        for k, val in zip(NAMES, theta):
            setattr(q, k, float(val))
        merger.set_params(q)
        _, loss, g = merger.backward(raw, info, target, weight=weight, out=out)
        return loss, g

    return fn


def params_of(base_params, theta):
    """base_params with the eight fitted values."""
    from . import params as P
    q = P.MergeParams(**vars(base_params))
    for k, val in zip(NAMES, theta):
        setattr(q, k, float(val))
    return q
