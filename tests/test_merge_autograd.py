"""The torch.autograd.Function of the test harness (tests/merge_autograd.py)
without a GPU: its wiring (the loss and gradient it passes to torch, the
chain rule through a reparametrisation, torch.optim.Adam steps) with a fake
Merger whose backward is a known quadratic; the GPU test of the real adjoint
through the same Function is in test_gpu_adjoint.py."""
import numpy as np
import torch

from imagestackalignator_b200 import params as P

from merge_autograd import NAMES, MergeLoss, MergeSetup

OPT = np.array([0.25, 3.0, 0.001, 0.006, 4.0, 2.0, 1.5, 0.12])
CURV = np.array([3.0, 0.5, 2e4, 5e3, 0.2, 0.7, 1.0, 40.0])


class FakeMerger:
    """backward(...) -> (None, loss, grad) of sum(CURV * (theta - OPT)^2) at the context's parameters."""

    def __init__(self, w, h, n, p):
        self.theta = np.array([getattr(p, k) for k in NAMES], np.float64)

    def backward(self, raw, info, target, weight=None):
        d = self.theta - OPT
        return None, float(np.sum(CURV * d * d)), 2 * CURV * d

    def close(self):
        pass


def _setup():
    return MergeSetup(FakeMerger, 64, 48, 3, P.MergeParams(), None, None, None, None)


def test_function_passes_loss_and_gradient():
    s = _setup()
    theta = torch.tensor(OPT * 1.2, dtype=torch.float64, requires_grad=True)
    loss = MergeLoss.apply(theta, s)
    loss.backward()
    d = OPT * 0.2
    assert np.isclose(loss.item(), np.sum(CURV * d * d))
    assert np.allclose(theta.grad.numpy(), 2 * CURV * d)
    # through a reparametrisation theta = base * s and a scaled loss
    u = torch.ones(8, dtype=torch.float64, requires_grad=True)
    (3.0 * MergeLoss.apply(torch.tensor(OPT * 1.2) * u, s)).backward()
    assert np.allclose(u.grad.numpy(), 3.0 * OPT * 1.2 * 2 * CURV * d)


def test_adam_through_the_function_converges():
    s = _setup()
    base = torch.tensor(OPT, dtype=torch.float64)
    u = torch.tensor([1.3, 0.8, 1.5, 1.2, 0.8, 1.25, 0.9, 1.3], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([u], lr=0.02)
    losses = []
    for _ in range(60):
        opt.zero_grad()
        loss = MergeLoss.apply(base * u, s)
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.2 * losses[0]
    assert s.calls == 60
