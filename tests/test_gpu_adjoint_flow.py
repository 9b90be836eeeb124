"""Gradient of the merge with respect to the tile flow and the eight merge
parameters (isa_merge_backward_tiles, sample mode BILINEAR) against FP64
central finite differences of the oracle merge (oracle/pipeline.py
merge_from_tiles), both evaluated at the same tile flows: the GPU's solved
ones plus a random 0.05-0.45 px (isa_tile_flow -> isa_set_tile_flow, and the
oracle's `tiles`). The offset keeps the flows off the integer shifts, where
the BILINEAR blend has kinks and a central difference averages the two
one-sided slopes (flat tiles sit exactly on them).

Burst: the differentiable-merge workload's statistics (10 frames, shifts up
to 6 px, rotations up to 0.2 degrees, noise a = 4e-4, b = 2e-6, merged at
1.5x) at 512 x 384, where the FP64 oracle's finite differences take seconds
each (at the full 4000 x 3000 one evaluation takes minutes). Loss: weighted
sum of squared differences of the merged image from a fixed target; the
weight excludes output pixels whose smallest weight sum is below 0.05
(ApplyWeighting's jump, as in test_gpu_adjoint).

The chain covers the accumulation and the robustness mask (through the
blended moved means), three LK iterations (warp, five-tap derivatives,
11 x 11 window sums, 2 x 2 solve) and the flow from tiles. The merge is
piecewise smooth in the flow (the warp's integer sample cell, the erosion's
minimum, the mask's clamps, |mr - mm|): a coordinate whose one-sided
differences over +-1e-6 px disagree by more than 1e-4 relative has a kink
inside the step and is counted, not compared. The adjoint is evaluated at
the GPU's FP32 forward (its LK flows differ from the FP64 oracle's by
~1e-5 px), so the bar is a relative error of 1e-3 on at least 90 % of the
compared coordinates and 2e-3 on all of them."""
import numpy as np
import pytest

import pipeline as PL
from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu

NCOORD = 32
BAR = 1e-3
NAMES = ["k_detail", "k_denoise", "dth", "dtr", "k_stretch", "k_shrink", "robust_s", "robust_t"]


@pytest.fixture(scope="module")
def case(cuda, oracle):
    import torch
    b = synthetic.make_burst(512, 384, 10, seed=21, max_shift=6.0, max_rot_deg=0.2, noise_a=4e-4, noise_b=2e-6)
    p = P.MergeParams()
    p.merge_scale = 1.5
    p.levels = P.default_levels(3)
    p.sample_mode = P.SAMPLE_BILINEAR
    m = isa.Merger(b.width, b.height, b.n, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    m.merge(raw, info)
    rng = np.random.default_rng(5)
    tiles = m.tile_flow(b.n).clone()
    tiles[1:] += torch.from_numpy(rng.uniform(0.05, 0.45, size=tuple(tiles[1:].shape)).astype(np.float32)).cuda()
    m.set_tile_flow(tiles)
    base = m.merge(raw, info).clone()
    torch.cuda.synchronize()
    t_np = tiles.cpu().numpy().astype(np.float64)
    tiles0 = {i: t_np[i].copy() for i in range(1, b.n)}
    keep = {}
    want = PL.merge_burst(b, p, lib=oracle, keep=keep, tiles=tiles0)
    return b, p, m, info, raw, base, tiles, tiles0, keep, want


def test_bilinear_forward_matches_oracle(case):
    """The BILINEAR merge on the GPU against the FP64 oracle at the same tile flows."""
    import torch
    b, p, m, info, raw, base, tiles, tiles0, keep, want = case
    out = m.merge(raw, info)
    torch.cuda.synchronize()
    assert torch.equal(out, base)  # the same tile flows, the same merge
    d = np.abs(out.cpu().numpy() - want.image)
    print("bilinear forward: max", d.max(), "p99.9", np.percentile(d, 99.9))
    assert np.percentile(d, 99.9) < 1e-4 and d.max() < 2e-3


def test_tile_flow_and_parameter_gradients_match_fp64_finite_differences(case, oracle):
    import torch
    b, p, m, info, raw, base, tiles, tiles0, keep, want = case
    target_np = (0.9 * base.cpu().numpy() + 0.03).astype(np.float32)
    target = torch.from_numpy(target_np).cuda()
    Wo, Ho = m.output_size(b.width, b.height)
    wsum = isa.device_copy(m.debug(0)["wsum"], (Ho, Wo, 3), torch.float32).cpu().numpy()
    om_np = (wsum.min(axis=2) > 0.05).astype(np.float32)
    om = torch.from_numpy(om_np).cuda()
    out, loss, grad, tg = m.backward_tiles(raw, info, target, weight=om)
    torch.cuda.synchronize()
    assert torch.equal(out, base)
    tg = tg.cpu().numpy().astype(np.float64)
    assert np.all(tg[0] == 0) and np.isfinite(tg).all()
    # the eight parameter gradients are those of the adjoint without the flow
    _, loss2, grad2 = m.backward(raw, info, target, weight=om)
    assert np.isclose(loss, loss2, rtol=1e-6) and np.allclose(grad, grad2, rtol=1e-4, atol=1e-9 * np.abs(grad2).max())
    om64 = om_np.astype(np.float64)[..., None]

    def oloss(tl, q=p):
        img = PL.merge_from_tiles(b, q, tl, keep, oracle).image
        return float(np.sum(om64 * (img - target_np) ** 2))

    l0 = oloss(tiles0)
    rng = np.random.default_rng(7)
    ty, tx = tg.shape[1:3]
    mag = np.abs(tg[1:]).reshape(-1)
    cand = np.flatnonzero(mag > 1e-3 * mag.max())  # tiles under the weighted image
    pick = rng.choice(cand, size=min(NCOORD, cand.size), replace=False)
    h = 1e-6
    rows = []
    for k in pick:
        i = 1 + k // (ty * tx * 2)
        r = k % (ty * tx * 2)
        y, x, c = r // (tx * 2), (r // 2) % tx, r % 2
        tp = {kk: v.copy() for kk, v in tiles0.items()}
        tm = {kk: v.copy() for kk, v in tiles0.items()}
        tp[i][y, x, c] += h
        tm[i][y, x, c] -= h
        lp, lm = oloss(tp), oloss(tm)
        fd, fwd, bwd = (lp - lm) / (2 * h), (lp - l0) / h, (l0 - lm) / h
        smooth = abs(fwd - bwd) <= 1e-4 * max(abs(fd), 1e-12)
        g = tg[i, y, x, c]
        rows.append((f"frame {i} tile ({y:2d},{x:2d}) c{c}", g, fd, abs(g - fd) / max(abs(fd), 1e-12), smooth))
    # the eight parameters, relative step 1e-4 in the FP32 values the GPU uses
    for k, name in enumerate(NAMES):
        v = float(getattr(p, name))
        pp, pm = P.MergeParams(**vars(p)), P.MergeParams(**vars(p))
        setattr(pp, name, float(np.float32(v + 1e-4 * abs(v))))
        setattr(pm, name, float(np.float32(v - 1e-4 * abs(v))))
        heff = float(np.float32(v + 1e-4 * abs(v))) - float(np.float32(v - 1e-4 * abs(v)))
        fd = (oloss(tiles0, pp) - oloss(tiles0, pm)) / heff
        rows.append((name, grad[k], fd, abs(grad[k] - fd) / max(abs(fd), 1e-12), True))
    print("\n".join(f"{n:28s} adjoint {g: .6e} fd {f: .6e} rel {e:.2e}{'' if s else '  kink'}" for n, g, f, e, s in rows))
    kinks = sum(not r[4] for r in rows)
    errs = np.array([r[3] for r in rows if r[4]])
    print(f"compared {errs.size}, kinks inside the step {kinks}; relative error median {np.median(errs):.2e}, "
          f"max {errs.max():.2e}, within {BAR:g}: {np.mean(errs <= BAR):.0%}")
    assert kinks <= NCOORD // 4
    assert np.mean(errs <= BAR) >= 0.9 and errs.max() <= 2 * BAR, rows
