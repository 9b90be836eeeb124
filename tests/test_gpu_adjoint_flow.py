"""Gradient of the merge with respect to the tile flow (isa_merge_backward_tiles,
sample mode BILINEAR) against FP64 central finite differences of the oracle
merge (oracle/pipeline.py merge_from_tiles), both evaluated at the GPU's own
tile flows (isa_tile_flow, offset by a random 0.05-0.45 px, -> isa_set_tile_flow
and the oracle's `tiles`). The offset keeps the flows off the integer shifts,
where the BILINEAR blend has kinks and a central difference averages the two
one-sided slopes.

Loss: weighted sum of squared differences of the merged image (scale 1.5)
from a fixed target; the weight excludes output pixels whose smallest
weight sum is below 0.05 (ApplyWeighting's jump, as in test_gpu_adjoint).
The chain covers the accumulation and the robustness mask (through the
blended moved means), three LK iterations (warp, five-tap derivatives,
11 x 11 window sums, 2 x 2 solve) and the flow from tiles. The merge is
piecewise smooth in the flow (the warp's integer sample cell, the erosion's
minimum, the mask's clamps, |mr - mm|), so the differences use a small step
(1e-5 px) and the bar is taken over the coordinates whose differences at
1e-5 and 1e-6 px agree to 1e-4 (no kink inside the step); those excluded
are counted and bounded. The adjoint is evaluated at the GPU's FP32 forward
(its LK flows differ from the FP64 oracle's by ~1e-5 px), so the bar is a
relative error of 1e-3 on at least 90 % of the checked coordinates and
2e-3 on all of them."""
import numpy as np
import pytest

import pipeline as PL
from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu

NCOORD = 32
BAR = 1e-3


@pytest.fixture(scope="module")
def case(cuda, oracle):
    import torch
    b = synthetic.make_burst(256, 192, 3, seed=21, max_shift=3.0, max_rot_deg=0.2)
    p = P.MergeParams()
    p.merge_scale = 1.5
    p.levels = P.default_levels(2)
    p.sample_mode = P.SAMPLE_BILINEAR
    m = isa.Merger(b.width, b.height, b.n, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    m.merge(raw, info)
    # the solved tile flows plus a sub-pixel offset: BILINEAR blends the integer shifts around the flow, so the merge
    # has a kink wherever a flow is an integer, which flat tiles (zero shift, no LK update) hit exactly
    rng = np.random.default_rng(5)
    tiles = m.tile_flow(b.n).clone()
    tiles[1:] += torch.from_numpy(rng.uniform(0.05, 0.45, size=tuple(tiles[1:].shape)).astype(np.float32)).cuda()
    m.set_tile_flow(tiles)
    base = m.merge(raw, info).clone()
    torch.cuda.synchronize()
    return b, p, m, info, raw, base, tiles


def test_bilinear_forward_matches_oracle(case, oracle):
    """The BILINEAR merge on the GPU against the FP64 oracle at the same tile flows."""
    import torch
    b, p, m, info, raw, base, tiles = case
    out = m.merge(raw, info)
    torch.cuda.synchronize()
    assert torch.equal(out, base)  # the same tile flows, the same merge
    t_np = tiles.cpu().numpy().astype(np.float64)
    want = PL.merge_burst(b, p, lib=oracle, tiles={i: t_np[i] for i in range(1, b.n)}).image
    d = np.abs(out.cpu().numpy() - want)
    print("bilinear forward: max", d.max(), "p99.9", np.percentile(d, 99.9))
    assert np.percentile(d, 99.9) < 1e-4 and d.max() < 2e-3


def test_tile_flow_gradient_matches_fp64_finite_differences(case, oracle):
    import torch
    b, p, m, info, raw, base, tiles = case
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
    # the eight scalar gradients are the plain adjoint's
    _, loss2, grad2 = m.backward(raw, info, target, weight=om)
    assert np.isclose(loss, loss2, rtol=1e-6) and np.allclose(grad, grad2, rtol=1e-4, atol=1e-9 * np.abs(grad2).max())

    t_np = tiles.cpu().numpy().astype(np.float64)
    tiles0 = {i: t_np[i].copy() for i in range(1, b.n)}
    keep = {}
    PL.merge_burst(b, p, lib=oracle, keep=keep, tiles=tiles0)
    om64 = om_np.astype(np.float64)[..., None]

    def oloss(tl):
        img = PL.merge_from_tiles(b, p, tl, keep, oracle).image
        return float(np.sum(om64 * (img - target_np) ** 2))

    def fd(i, y, x, c, h):
        tp = {k: v.copy() for k, v in tiles0.items()}
        tm = {k: v.copy() for k, v in tiles0.items()}
        tp[i][y, x, c] += h
        tm[i][y, x, c] -= h
        return (oloss(tp) - oloss(tm)) / (2 * h)

    rng = np.random.default_rng(7)
    ty, tx = t_np.shape[1:3]
    # coordinates with a gradient clear of zero (the tiles under the weighted image)
    mag = np.abs(tg[1:]).reshape(-1)
    cand = np.flatnonzero(mag > 1e-3 * mag.max())
    pick = rng.choice(cand, size=min(NCOORD, cand.size), replace=False)
    rows, checked, kinks = [], 0, 0
    for k in pick:
        i = 1 + k // (ty * tx * 2)
        r = k % (ty * tx * 2)
        y, x, c = r // (tx * 2), (r // 2) % tx, r % 2
        f5, f6 = fd(i, y, x, c, 1e-5), fd(i, y, x, c, 1e-6)
        g = tg[i, y, x, c]
        smooth = abs(f5 - f6) <= 1e-4 * max(abs(f5), 1e-12)
        err = abs(g - f5) / max(abs(f5), 1e-12)
        rows.append((i, y, x, c, g, f5, f6, err, smooth))
        if smooth:
            checked += 1
        else:
            kinks += 1
    print("\n".join(f"frame {i} tile ({y:2d},{x:2d}) c{c}: adjoint {g: .6e} fd {f5: .6e} ({f6: .6e}) rel {e:.2e}{'' if s else '  kink'}"
                    for i, y, x, c, g, f5, f6, e, s in rows))
    print(f"checked {checked}, kinks inside the step {kinks}")
    assert kinks <= len(rows) // 4
    errs = np.array([r[7] for r in rows if r[8]])
    print(f"relative error: median {np.median(errs):.2e}, max {errs.max():.2e}, within {BAR:g}: {np.mean(errs <= BAR):.0%}")
    assert np.mean(errs <= BAR) >= 0.9 and errs.max() <= 2 * BAR, rows
