"""Sample mode BILINEAR in the FP64 oracle (oracle/isa_oracle.c accumulate_mode
and robustness_mask_mode, oracle/pipeline.py): equal to ROUND where the flow
puts every frame on an integer shift, continuous in the tile flow elsewhere,
and merge_from_tiles reproduces merge_burst at the same tile flows (to FP64
rounding: it adds the frames' sums in frame order)."""
import numpy as np
import pytest

from imagestackalignator_b200 import params as P, synthetic

import pipeline as PL


@pytest.fixture(scope="module")
def bil(oracle):
    b = synthetic.make_burst(160, 128, 3, seed=5, max_shift=3.0, max_rot_deg=0.2)
    p = P.MergeParams()
    p.merge_scale = 1.5
    p.levels = P.default_levels(2)
    p.sample_mode = P.SAMPLE_BILINEAR
    keep = {}
    res = PL.merge_burst(b, p, lib=oracle, keep=keep)
    return b, p, keep, res


def test_merge_from_tiles_reproduces_merge_burst(bil, oracle):
    b, p, keep, res = bil
    again = PL.merge_from_tiles(b, p, keep["tiles"], keep, oracle)
    np.testing.assert_allclose(again.image, res.image, rtol=0, atol=1e-12)
    twice = PL.merge_from_tiles(b, p, keep["tiles"], keep, oracle)  # from the cache
    np.testing.assert_array_equal(twice.image, again.image)


def test_bilinear_equals_round_at_integer_shifts(bil, oracle):
    """A constant flow of even integers per frame puts the accumulation (s = 2) and the mask (flow / 2) on
    integer shifts (its bilinear samples are exact)."""
    b, p, keep, res = bil
    n, H, W = b.raw.shape
    q = P.MergeParams(**vars(p))
    q.merge_scale = 2.0
    rng = np.random.default_rng(3)
    flows = {i: np.broadcast_to(2.0 * rng.integers(-2, 3, size=2), (H, W, 2)).astype(np.float64) for i in range(1, n)}
    white = np.asarray(b.white, np.float64)
    black = np.asarray(b.black, np.float64)
    max_val = float(np.max(np.float32(white) + np.float32(black)))
    ref_half = oracle.debayer_subsample(b.raw[0], b.cfa, max_val)
    out = {}
    for mode in (P.SAMPLE_ROUND, P.SAMPLE_BILINEAR):
        q.sample_mode = mode
        masks = {}
        for i in range(1, n):
            mov = oracle.debayer_subsample(b.raw[i], b.cfa, max_val)
            m = oracle.robustness_mask(ref_half, mov, flows[i], float(np.float32(b.noise_a)), float(np.float32(b.noise_b)),
                                       q.f32("threshold_m"), np.ones((H // 2, W // 2, 4)), q.f32("robust_s"), q.f32("robust_t"),
                                       bilinear=mode == P.SAMPLE_BILINEAR)
            masks[i] = oracle.erode(m, q.erode_size)
        out[mode] = PL.merge_tail(b, q, flows, masks, keep["kparam"], oracle).image
    np.testing.assert_array_equal(out[P.SAMPLE_ROUND], out[P.SAMPLE_BILINEAR])


def test_bilinear_loss_is_continuous_in_the_tile_flow(bil, oracle):
    """Central differences at 1e-5 and 1e-6 px agree (no jump inside the step) and are not all zero."""
    b, p, keep, res = bil
    tgt = 0.9 * res.image + 0.03
    om = (res.wsum.min(axis=2) > 0.05).astype(np.float64)[..., None]

    def loss(tl):
        return float(np.sum(om * (PL.merge_from_tiles(b, p, tl, keep, oracle).image - tgt) ** 2))

    rng = np.random.default_rng(1)
    ty, tx = keep["tiles"][1].shape[:2]
    agree, nonzero = 0, 0
    for _ in range(4):
        i, y, x, c = int(rng.integers(1, b.n)), int(rng.integers(ty)), int(rng.integers(tx)), int(rng.integers(2))
        d = []
        for h in (1e-5, 1e-6):
            tp = {k: v.copy() for k, v in keep["tiles"].items()}
            tm = {k: v.copy() for k, v in keep["tiles"].items()}
            tp[i][y, x, c] += h
            tm[i][y, x, c] -= h
            d.append((loss(tp) - loss(tm)) / (2 * h))
        agree += abs(d[0] - d[1]) <= 1e-3 * max(abs(d[0]), 1e-12)
        nonzero += d[0] != 0.0
    assert agree >= 3 and nonzero >= 3


def test_merge_from_tiles_follows_parameter_changes(bil, oracle):
    """Its caches are keyed on what each step depends on: a change of the
    kernel-shape or robustness parameters gives the full merge's image."""
    b, p, keep, res = bil
    PL.merge_from_tiles(b, p, keep["tiles"], keep, oracle)  # fill the caches at p
    for name, factor in (("k_detail", 1.2), ("robust_t", 0.8)):
        q = P.MergeParams(**vars(p))
        setattr(q, name, float(np.float32(getattr(p, name) * factor)))
        want = PL.merge_burst(b, q, lib=oracle, tiles=keep["tiles"]).image
        got = PL.merge_from_tiles(b, q, keep["tiles"], keep, oracle).image
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
        assert np.abs(got - res.image).max() > 1e-6  # the change is visible
