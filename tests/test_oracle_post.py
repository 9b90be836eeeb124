"""Colour/tone post-processing and TIFF output without a GPU: the oracle's
gamma against golden vectors of the reference's own FP32 GammasRGB, the host
entry points of libisa.so (isa_color_twists, isa_save_tiff16) against the
oracle bit for bit, the LUT cubic's properties, and the argument checks of
isa_postprocess (rejected before any CUDA call)."""
import ctypes
import os

import numpy as np
import pytest

from imagestackalignator_b200 import isa

import post as PO

HERE = os.path.dirname(os.path.abspath(__file__))


def lut_levels():
    """The controller's LUTx: 256 levels i / 255 written with nine decimals."""
    return np.float32(np.round(np.arange(256) / 255.0, 9))


def s_curve(x):
    x = np.asarray(x, np.float64)
    return np.float32(x + 0.15 * np.sin(2 * np.pi * x) / (2 * np.pi))


def test_gamma_matches_reference_golden():
    g = np.load(os.path.join(HERE, "golden", "post_golden.npz"))
    assert np.array_equal(PO.gamma_srgb(g["in_gamma32"]), g["out_gamma32"])


def test_gamma_live_reference_when_present():
    path = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref32.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    import pipeline as PL
    v = np.random.default_rng(3).random((32, 40, 3)).astype(np.float32) * np.float32(1.5) - np.float32(0.2)
    assert np.array_equal(PO.gamma_srgb(v), PL.StageLib("ref32").gamma_srgb(v))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_color_twists_match_oracle(seed):
    rng = np.random.default_rng(seed)
    cam = np.eye(3) * 0.7 + rng.random((3, 3)) * 0.2
    t1, t2 = isa.color_twists(cam)
    o1, o2 = PO.color_twists(cam)
    assert np.array_equal(t1, o1) and np.array_equal(t2, o2)
    assert np.all(t1[:, 3] == 0) and np.all(t2[:, 3] == 0)
    # ProPhoto -> sRGB maps the D50 white of one space to the other's: rows sum to 1 up to float rounding
    assert np.allclose(t2[:, :3].sum(1), 1.0, atol=1e-5)


def test_color_twists_identity_chain():
    """Camera = ProPhoto's own toPCS: twist1 is the identity (to FP64 rounding, then float)."""
    pp_to, _ = PO._color_space(PO.PROPHOTO)
    t1, _ = isa.color_twists(np.array(pp_to))
    assert np.allclose(t1[:, :3], np.eye(3), atol=1e-6)


@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (37, 53), (64, 17)])
def test_tiff_bytes_match_oracle(tmp_path, shape):
    h, w = shape
    rgb = np.random.default_rng(h * 100 + w).integers(0, 65536, (h, w, 3), dtype=np.uint16)
    path = tmp_path / "out.tif"
    isa.save_tiff16(str(path), rgb)
    buf = path.read_bytes()
    assert buf == PO.tiff16_bytes(rgb)
    tags, img = PO.parse_tiff16(buf)
    assert np.array_equal(img, rgb)
    assert tags[256][2] == w and tags[257][2] == h and tags[258][1] == 3 and tags[277][2] == 3
    assert tags[273][2] == 200 and tags[279][2] == w * h * 6 and len(buf) == 200 + w * h * 6
    assert buf[tags[271][2]:tags[271][2] + 8] == b"MK TIFF\0"


def test_tiff_rejects_bad_arguments(tmp_path):
    rgb = np.zeros((2, 2, 3), np.uint16)
    lib = isa.lib()
    assert lib.isa_save_tiff16(None, rgb.ctypes.data_as(ctypes.c_void_p), 2, 2) == isa.ISA_EINVAL
    assert lib.isa_save_tiff16(os.fsencode(str(tmp_path / "x.tif")), rgb.ctypes.data_as(ctypes.c_void_p), 0, 2) == isa.ISA_EINVAL
    assert lib.isa_save_tiff16(os.fsencode(str(tmp_path / "no" / "dir" / "x.tif")), rgb.ctypes.data_as(ctypes.c_void_p), 2, 2) == isa.ISA_EINVAL


def test_lut_cubic_properties():
    lx = lut_levels()
    ly = s_curve(lx)
    # at the levels the cubic returns the table value exactly
    assert np.array_equal(PO.lut_cubic(lx, ly, lx), ly)
    # a cubic table is reproduced to float rounding
    v = np.random.default_rng(4).random(5000).astype(np.float32)
    cub = lambda x: np.float32(0.2 + 0.5 * np.asarray(x, np.float64) - 0.3 * np.asarray(x, np.float64) ** 3)
    assert np.abs(PO.lut_cubic(lx, cub(lx), v).astype(np.float64) - cub(v)).max() < 2e-6
    # segments: the largest level not above the value, capped at n - 2; NaN -> 0
    k = PO.lut_segment(lx, np.array([0.0, lx[5], np.nextafter(lx[5], np.float32(0)), 1.0, np.nan], np.float32))
    assert list(k) == [0, 5, 4, 254, 0]


def _pp(crop=(0, 0, 4, 4), nlut=8, lx=None):
    lx = np.linspace(0, 1, nlut).astype(np.float32) if lx is None else lx
    t = np.zeros((3, 4), np.float32)
    return isa.post_params(crop, [1, 1, 1], t, t, lx, lx, 0.0)


def test_postprocess_argument_checks():
    lib = isa.lib()
    fake = ctypes.c_void_p(256)
    cases = [
        (_pp(crop=(0, 0, 5, 4)), 0),       # crop wider than the image
        (_pp(crop=(-1, 0, 2, 2)), 0),
        (_pp(nlut=3), 0),                  # too few levels
        (_pp(lx=np.array([0, 0.5, 0.5, 1], np.float32)), 0),  # not increasing
        (_pp(), 7),                        # unknown format
    ]
    for (pp, keep), fmt in cases:
        rc = lib.isa_postprocess(fake, ctypes.c_size_t(4 * 12), 4, 4, ctypes.byref(pp), fmt, fake, ctypes.c_size_t(64), None)
        assert rc == isa.ISA_EINVAL, (fmt, rc)
    pp, keep = _pp()
    assert lib.isa_postprocess(None, ctypes.c_size_t(48), 4, 4, ctypes.byref(pp), 0, fake, ctypes.c_size_t(64), None) == isa.ISA_EINVAL
    assert lib.isa_postprocess(fake, ctypes.c_size_t(47), 4, 4, ctypes.byref(pp), 0, fake, ctypes.c_size_t(64), None) == isa.ISA_EINVAL
    assert lib.isa_postprocess(fake, ctypes.c_size_t(48), 4, 4, ctypes.byref(pp), 0, fake, ctypes.c_size_t(20), None) == isa.ISA_EINVAL


def test_postprocess_oracle_edge_values():
    """The restatement on values that exercise every clamp: NaN and +-inf give 0 after
    the gamma, negatives 0, and values above the camera white saturate."""
    lx = lut_levels()
    t1, t2 = PO.color_twists(np.eye(3) * 0.9)
    img = np.array([[[np.nan, 0.5, 0.2], [np.inf, -np.inf, 0.0], [-1.0, 2.0, 0.7], [0.3, 0.3, 0.3]]], np.float32)
    out = PO.postprocess(img, (0, 0, 4, 1), [1.0, 0.8, 1.2], t1, t2, lx, lx, 0.0)
    assert out.dtype == np.uint16 and out.shape == (1, 4, 3)
    bgra = PO.postprocess(img, (0, 0, 4, 1), [1.0, 0.8, 1.2], t1, t2, lx, lx, 0.0, fmt=1)
    assert bgra.dtype == np.uint8 and np.all(bgra[..., 3] == 255)
    assert np.array_equal(bgra[..., 0], np.clip(np.rint(bgra[..., 0]), 0, 255))
