"""Whole-pipeline checks of the CPU oracle: known-answer tests regenerated from
the mathematics (the reference's own manual checks, TestCC and the seeded
TestRawFile scene, ImageStackAlignatorController.cs:1389-1449 and
TestRawFile.cs:39-64), and the restatement against the reference kernels run
end to end."""
import os

import numpy as np
import pytest
from scipy.ndimage import uniform_filter

from imagestackalignator_b200 import params as P, synthetic

import pipeline as PL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def texture_burst(W=512, H=384, shifts=((0, 0), (4, 2), (-6, 10)), seed=0):
    """TestRawFile-style scene: seeded uniform noise, box-blurred, moved by
    known even shifts (even so the CFA phase is kept)."""
    rng = np.random.default_rng(seed)
    tex = uniform_filter(rng.uniform(0, 1, (H + 64, W + 64)), 5)
    tex = (tex - tex.min()) / (tex.max() - tex.min())
    b = synthetic.make_burst(W, H, len(shifts), seed=seed, max_shift=0, max_rot_deg=0)
    for i, (dx, dy) in enumerate(shifts):
        t = tex[32 - dy:32 - dy + H, 32 - dx:32 - dx + W]
        b.raw[i] = np.round(512 + t * 15000).astype(np.uint16)
    return b


def test_known_integer_shifts_are_recovered(oracle):
    shifts = ((0, 0), (4, 2), (-6, 10))
    b = texture_burst(shifts=shifts)
    keep = {}
    PL.merge_burst(b, P.MergeParams(), lib=oracle, keep=keep)
    for i in (1, 2):
        fl = keep["flow"][i][24:-24, 24:-24].reshape(-1, 2)
        med = np.median(fl, axis=0)
        np.testing.assert_allclose(med, shifts[i], atol=1e-3)
        # the integer shift the accumulation uses is exact almost everywhere
        assert (np.round(fl) == np.array(shifts[i])).all(axis=1).mean() > 0.99
        tiles = keep["tiles"][i].reshape(-1, 2)
        assert (np.abs(np.median(tiles, axis=0) - shifts[i]) < 0.25).all()


def test_identical_frames_merge_to_the_reference_frame_accumulation(oracle):
    b = texture_burst(shifts=((0, 0), (0, 0), (0, 0)))
    keep = {}
    p = P.MergeParams()
    p.merge_scale = 1.0  # no fallback blend (the plain mode's threshold 1 depends on the frame count)
    r = PL.merge_burst(b, p, lib=oracle, keep=keep)
    for i in (1, 2):
        # the sub-pixel fit of the tile search (kernel.cu:475-540) is not exactly
        # zero on identical tiles, and LK (which leaves the h-wide border alone)
        # only shrinks it; in the interior it rounds to 0
        assert np.abs(keep["flow"][i][8:-8, 8:-8]).max() < 0.5
        assert (keep["mask"][i][4:-4, 4:-4, :3] == 1.0).all()
    # one frame alone, same kernel: the merge of identical frames has the same ratio
    single = synthetic.Burst(raw=b.raw[:2].copy(), cfa=b.cfa, black=b.black, white=b.white, noise_a=b.noise_a, noise_b=b.noise_b,
                             shifts=b.shifts[:2], rotations=b.rotations[:2])
    r1 = PL.merge_burst(single, p, lib=oracle)
    np.testing.assert_allclose(r.image[12:-12, 12:-12], r1.image[12:-12, 12:-12], rtol=0, atol=1e-12)


def test_merge_modes_have_the_reference_geometry(oracle, small_burst):
    for mode, shape in (("plain", (384, 512, 3)), ("super", (384, 512, 3)), ("x2", (768, 1024, 3))):
        p = P.MergeParams()
        p.super_resolution = mode == "super"
        p.merge_scale = 2.0 if mode == "x2" else 0.0
        r = PL.merge_burst(small_burst, p, lib=oracle)
        assert r.image.shape == shape
        assert np.isfinite(r.image).all()
        inner = r.image[8:-8, 8:-8]
        assert -0.1 <= inner.min() and inner.max() <= 1.1  # noise around black and white is kept (no clipping in the merge)


@pytest.mark.parametrize("mode", ["plain", "x2"])
def test_restatement_matches_reference_kernels_end_to_end(oracle, mode):
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref64.so")):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    b = synthetic.make_burst(256, 192, 5, seed=11, max_shift=4, max_rot_deg=0.2)
    p = P.MergeParams()
    p.levels = P.default_levels(3)
    if mode == "x2":
        p.merge_scale = 2.0
    mine = PL.merge_burst(b, p, lib=oracle)
    ref = PL.merge_burst(b, p, kind="ref64")
    np.testing.assert_allclose(mine.image, ref.image, rtol=0, atol=1e-9)
