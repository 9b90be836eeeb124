"""Adjoint of the merge (isa_merge_backward) against FP64 central finite
differences of the oracle merge, for the eight merge parameters: the kernel
shape (k_detail, k_denoise, dth, dtr, k_stretch, k_shrink) and the
robustness mask (robust_s, robust_t). Loss: weighted sum of squared
differences of the merged image from a fixed target, on a small burst merged
at scale 1.5, step 1e-4 relative.

The merged image jumps where a channel's certainty-weighted weight sum
reaches zero (ApplyWeighting outputs 0 there), and many output pixels of
strongly anisotropic kernels have such sums near zero; the loss weight
excludes pixels whose smallest weight sum is below 0.05 at the evaluation
point, so that the finite differences see the smooth piece the adjoint
differentiates. The GPU evaluates the gradient at its own FP32 forward; the
two forwards take different integer shifts at a few pixels whose flow sits
at a rounding boundary."""
import numpy as np
import pytest

import pipeline as PL
from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu

NAMES = ["k_detail", "k_denoise", "dth", "dtr", "k_stretch", "k_shrink", "robust_s", "robust_t"]


@pytest.fixture(scope="module")
def setup():
    b = synthetic.make_burst(384, 320, 3, seed=11, max_shift=4.0, max_rot_deg=0.2)
    p = P.MergeParams()
    p.merge_scale = 1.5
    return b, p


def oracle_loss(oracle, b, p, target, om):
    img = PL.merge_burst(b, p, lib=oracle).image
    return float(np.sum(om[..., None] * (img - target) ** 2))


def test_gradient_matches_fp64_finite_differences(cuda, oracle, setup):
    import torch
    b, p = setup
    m = isa.Merger(b.width, b.height, b.n, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    base = m.merge(raw, info)
    torch.cuda.synchronize()
    target_np = (0.9 * base.cpu().numpy() + 0.03).astype(np.float32)
    target = torch.from_numpy(target_np).cuda()
    Wo, Ho = m.output_size(b.width, b.height)
    wsum = isa.device_copy(m.debug(0)["wsum"], (Ho, Wo, 3), torch.float32).cpu().numpy()
    om_np = (wsum.min(axis=2) > 0.05).astype(np.float32)
    om = torch.from_numpy(om_np).cuda()
    out, loss, grad = m.backward(raw, info, target, weight=om)
    torch.cuda.synchronize()
    assert torch.equal(out, base)  # the forward inside the adjoint is the merge
    want_loss = float(np.sum(om_np[..., None].astype(np.float64) * (base.cpu().numpy().astype(np.float64) - target_np) ** 2))
    np.testing.assert_allclose(loss, want_loss, rtol=1e-6)
    errs = []
    for k, name in enumerate(NAMES):
        v = float(getattr(p, name))
        h = 1e-4 * abs(v)
        pp, pm = P.MergeParams(**vars(p)), P.MergeParams(**vars(p))
        setattr(pp, name, float(np.float32(v + h)))
        setattr(pm, name, float(np.float32(v - h)))
        heff = float(np.float32(v + h)) - float(np.float32(v - h))
        fd = (oracle_loss(oracle, b, pp, target_np, om_np) - oracle_loss(oracle, b, pm, target_np, om_np)) / heff
        err = abs(grad[k] - fd) / max(abs(fd), 1e-12)
        errs.append((name, grad[k], fd, err))
    print("\n".join(f"{n:10s} adjoint {g: .6e}  fd {f: .6e}  rel {e:.2e}" for n, g, f, e in errs))
    for name, g, f, e in errs:
        assert e <= 1e-3, (name, g, f, e)
    m.close()


def test_adam_fit_lowers_the_loss(cuda, setup):
    """A few Adam steps on the eight parameters from a perturbed start move
    the merge toward the target made with the defaults."""
    import torch
    b, p0 = setup
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    m0 = isa.Merger(b.width, b.height, b.n, p0)
    target = m0.merge(raw, info).clone()
    torch.cuda.synchronize()
    Wo, Ho = m0.output_size(b.width, b.height)
    wsum = isa.device_copy(m0.debug(0)["wsum"], (Ho, Wo, 3), torch.float32)
    om = (wsum.min(dim=2).values > 0.05).float().contiguous()
    m0.close()
    theta = np.array([getattr(p0, n) for n in NAMES], np.float64) * np.array([1.3, 0.8, 1.5, 1.2, 0.8, 1.25, 0.9, 1.3])
    lr = 0.02 * np.abs(theta)
    mom, vel = np.zeros(8), np.zeros(8)
    losses = []
    for step in range(1, 16):
        p = P.MergeParams(**vars(p0))
        for n, v in zip(NAMES, theta):
            setattr(p, n, float(v))
        m = isa.Merger(b.width, b.height, b.n, p)
        _, loss, g = m.backward(raw, info, target, weight=om)
        m.close()
        losses.append(loss)
        mom = 0.9 * mom + 0.1 * g
        vel = 0.999 * vel + 0.001 * g * g
        theta = theta - lr * (mom / (1 - 0.9 ** step)) / (np.sqrt(vel / (1 - 0.999 ** step)) + 1e-30)
    assert losses[-1] < 0.5 * losses[0], losses


def test_autograd_function_adam_fit(cuda, setup):
    """The same fit through the harness's torch.autograd.Function (tests/merge_autograd.py)
    and torch.optim.Adam on per-parameter factors; the Function's first gradient is the
    adjoint's own."""
    import torch
    from merge_autograd import MergeLoss, MergeSetup
    b, p0 = setup
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    m0 = isa.Merger(b.width, b.height, b.n, p0)
    target = m0.merge(raw, info).clone()
    torch.cuda.synchronize()
    Wo, Ho = m0.output_size(b.width, b.height)
    wsum = isa.device_copy(m0.debug(0)["wsum"], (Ho, Wo, 3), torch.float32)
    om = (wsum.min(dim=2).values > 0.05).float().contiguous()
    m0.close()
    s = MergeSetup(isa.Merger, b.width, b.height, b.n, p0, raw, info, target, om)
    base = torch.tensor([getattr(p0, n) for n in NAMES], dtype=torch.float64)
    u = torch.tensor([1.3, 0.8, 1.5, 1.2, 0.8, 1.25, 0.9, 1.3], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([u], lr=0.02, eps=1e-30)
    losses = []
    for step in range(15):
        opt.zero_grad()
        loss = MergeLoss.apply(base * u, s)
        loss.backward()
        if step == 0:
            p = s.params((base * u).detach().numpy())
            m = isa.Merger(b.width, b.height, b.n, p)
            _, l0, g0 = m.backward(raw, info, target, weight=om)
            m.close()
            # a second adjoint call: its float atomics may sum in another order
            assert np.isclose(l0, loss.item(), rtol=1e-5, atol=0)
            want = base.numpy() * g0
            assert np.allclose(u.grad.numpy(), want, rtol=1e-3, atol=1e-6 * np.abs(want).max())
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.5 * losses[0], losses
