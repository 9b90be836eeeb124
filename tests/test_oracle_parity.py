"""The decision-aware parity checker (oracle/parity.py) on CPU: it must pass an
exact copy of the oracle's merge, exclude exactly the pixels that read a
planted differing decision, and fail on planted errors elsewhere."""
import numpy as np
import pytest

from imagestackalignator_b200 import params as P, synthetic

import parity
import pipeline as PL


@pytest.fixture(scope="module")
def merged(oracle):
    b = synthetic.make_burst(192, 128, 3, seed=4, max_shift=3, max_rot_deg=0.1)
    p = P.MergeParams()
    p.levels = P.default_levels(2)
    keep = {}
    res = PL.merge_burst(b, p, lib=oracle, keep=keep)
    return b, p, keep, res


def _args(b, p, keep):
    flows = {i: keep["flow"][i].copy() for i in keep["flow"]}
    masks = {i: keep["mask"][i].copy() for i in keep["mask"]}
    return flows, masks, PL.out_geometry(b.width, b.height, p)


def test_identical_merge_passes(merged):
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    st = parity.merge_parity(res.image.copy(), res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size,
                             wsum_orc=res.wsum)
    assert st["max_abs_matched"] == 0.0 and st["excluded_shift"] == 0 and st["mask_cells_differ"] == 0


def test_planted_pixel_error_fails(merged):
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    got = res.image.copy()
    got[40, 50, 1] += 2e-4
    with pytest.raises(AssertionError, match="decision-matched"):
        parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum)


def test_flipped_shift_decision_is_excluded(merged):
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    y, x = 60, 70
    f = flows[1][y, x, 0]
    flows[1][y, x, 0] = np.floor(f + 0.5) + 0.6  # rounds one integer higher than the oracle's flow
    got = res.image.copy()
    got[y, x] += 0.05
    st = parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum)
    assert st["excluded_shift"] >= 1 and st["max_abs_matched"] == 0.0


def test_unexplained_mask_difference_fails(merged):
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    masks[2][30, 40, 0] = masks[2][30, 40, 0] * 0.5 + 0.25
    with pytest.raises(AssertionError, match="no differing rounding decision"):
        parity.merge_parity(res.image.copy(), res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum)


def test_explained_mask_difference_is_excluded(merged):
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    hy, hx = 30, 40
    # the mask offset round(flow / 2) at half-res cell (hx, hy) samples the flow between pixels 2hx..2hx+1, 2hy..2hy+1
    for yy in (2 * hy, 2 * hy + 1):
        for xx in (2 * hx, 2 * hx + 1):
            flows[2][yy, xx, 0] += 2.0
    masks[2][hy, hx + 1, 0] += 0.3
    got = res.image.copy()
    got[2 * hy, 2 * hx + 2] += 0.01
    st = parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum)
    assert st["mask_cells_differ"] == 1 and st["excluded_mask"] > 0 and st["max_abs_matched"] == 0.0


def test_track_parity_on_the_oracles_own_record(merged):
    """A record built from the oracle's own argmins and offsets passes; a
    changed argmin outside a tie fails."""
    b, p, keep, res = merged
    pairs = P.shift_pairs(b.n, 0, p.tracking_strategy, p.tracking_block_size)
    parts = []
    for li, lv in enumerate(p.levels):
        am = [np.argmin(keep["scores"][(li, r, t)], axis=1) for (r, t) in pairs]
        of = [parity.c_round(keep["offsets"][(li, r, t)]).astype(np.int64) for (r, t) in pairs]
        parts += [np.concatenate(am), np.concatenate(of).reshape(-1)]
    rec = np.concatenate(parts).astype(np.int32)
    st = parity.track_parity(rec, keep, pairs, p.levels, b.width, b.height)
    assert st["argmin_checked"] == st["tiles"] and st["offset_flips"] == 0
    sc = keep["scores"][(0, pairs[0][0], pairs[0][1])]
    srt = np.sort(sc, axis=1)
    j = int(np.argmax((srt[:, 1] - srt[:, 0]) / np.maximum(srt[:, 0], 1e-30)))  # the clearest minimum
    bad = rec.copy()
    bad[j] = (bad[j] + 1) % sc.shape[1]
    with pytest.raises(AssertionError, match="integer shift"):
        parity.track_parity(bad, keep, pairs, p.levels, b.width, b.height)


def test_weight_threshold_decision_is_identified(merged):
    """ApplyWeighting's w < 1 (plain merge): a channel whose weight sum lies on
    the other side of the threshold on the GPU is excluded, wherever it is."""
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    wg = res.wsum.copy()
    y, x = 50, 90
    wg[y, x, 1] = 0.99999 if res.wsum[y, x, 1] >= 1 else 1.00001
    got = res.image.copy()
    got[y, x, 1] += 1e-3
    st = parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum,
                             wsum_gpu=wg)
    assert st["excluded_weight"] == 1 and st["max_abs_matched"] == 0.0
    got[y + 1, x, 1] += 1e-3
    with pytest.raises(AssertionError, match="decision-matched"):
        parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum, wsum_gpu=wg)



def test_substituted_tail_explains_upstream_differences(merged, oracle):
    """A pixel off by more than the bar is counted as carried in from upstream
    when the oracle's accumulation fed the same flows and masks reproduces
    it; an error of the accumulation itself still fails."""
    b, p, keep, res = merged
    flows, masks, geom = _args(b, p, keep)
    masks[1][20, 30, 2] = max(masks[1][20, 30, 2] - 5e-6, 0.0)  # within the mask tolerance
    sub = PL.merge_tail(b, p, flows, masks, keep["kparam"], oracle)
    got = sub.image.copy()
    y, x = 41, 61
    got[y, x] = res.image[y, x] + 3e-4          # upstream: the substituted oracle moves with it
    sub.image[y, x] = got[y, x]
    st = parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum,
                             want_sub=sub.image, wsum_sub=sub.wsum)
    assert st["excluded_conditioned"] >= 1 and st["tail_max_abs"] <= parity.IMAGE_BAR
    got[y + 2, x] += 3e-4                        # not reproduced by the substituted oracle: the accumulation's own error
    with pytest.raises(AssertionError, match="own flows, masks and kernel parameters"):
        parity.merge_parity(got, res.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=res.wsum,
                            want_sub=sub.image)


def test_merge_tail_reproduces_the_oracle(merged, oracle):
    b, p, keep, res = merged
    sub = PL.merge_tail(b, p, keep["flow"], keep["mask"], keep["kparam"], oracle)
    np.testing.assert_array_equal(sub.image, res.image)
