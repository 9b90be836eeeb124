"""DNG pixel data on the GPU (isa_dng_decode) against the restated reference
reader (oracle/raw.py over orc_dng_decode), bit-exact: lossless-JPEG tiles
with every predictor and one or two interleaved components, strips,
restart markers, tiles that overhang the frame, linearisation and black-
level deltas, a sample above the bit depth (the reference stops), and
uncompressed 16-bit and packed strips."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa

import raw as R

pytestmark = pytest.mark.gpu


def run(file, W, H, offs, cnts, **kw):
    import torch
    out = isa.dng_decode(file, W, H, offs, cnts, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("psv", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("clrs", [1, 2])
def test_lj92_tiles(cuda, psv, clrs):
    rng = np.random.default_rng(psv * 10 + clrs)
    H, W = 100, 160
    img = np.clip(rng.normal(3000, 500, (H, W)), 0, 16383).astype(np.uint16)
    f, offs, cnts = R.dng_tiles(img, 64, 48, clrs=clrs, bits=14, psv=psv)
    kw = dict(tiled=True, tile_w=64, tile_h=48)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)


def test_lj92_strips_restart_lin_black(cuda):
    rng = np.random.default_rng(3)
    H, W = 90, 128
    img = np.clip(rng.normal(2000, 400, (H, W)), 0, 4095).astype(np.uint16)
    parts, offs, cnts, pos = [np.zeros(16, np.uint8)], [], [], 16
    rps = 30
    for s in range(0, H, rps):
        t = R.lj92_encode(img[s:s + rps], clrs=2, bits=12, psv=1, restart=64 * 10)
        offs.append(pos); cnts.append(len(t)); parts.append(t); pos += len(t)
    f = np.concatenate(parts)
    lin = (np.arange(4096) * 3 // 2).astype(np.uint16)
    bh = rng.integers(0, 40, W).astype(np.uint16)
    bv = rng.integers(0, 40, H).astype(np.uint16)
    kw = dict(tiled=False, rows_per_strip=rps, linearization=lin, black_h=bh, black_v=bv)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)


def test_lj92_overhanging_tiles_and_large_frame(cuda):
    rng = np.random.default_rng(4)
    H, W = 600, 1000                  # tiles of 256 overhang both edges
    img = np.clip(rng.normal(8000, 900, (H, W)), 0, 16383).astype(np.uint16)
    f, offs, cnts = R.dng_tiles(img, 256, 256, clrs=2, bits=14, psv=1)
    kw = dict(tiled=True, tile_w=256, tile_h=256)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)


def test_lj92_sample_above_bit_depth_is_an_error(cuda):
    img = np.full((16, 32), 5000, np.uint16)
    f, offs, cnts = R.dng_tiles(img, 32, 16, clrs=1, bits=14, psv=1)
    # declare 12 bits in the frame header (SOF3 precision byte follows the 4-byte marker/length after SOI)
    g = f.copy()
    sof = 32 + 2
    assert g[sof] == 0xFF and g[sof + 1] == 0xC3
    g[sof + 4] = 12
    st, _ = R.dng_decode(g, 32, 16, offs, cnts, tiled=True, tile_w=32, tile_h=16)
    assert st == -1
    with pytest.raises(isa.IsaError):
        run(g, 32, 16, offs, cnts, tiled=True, tile_w=32, tile_h=16)


@pytest.mark.parametrize("depth", [16, 14, 12, 10])
def test_uncompressed_strips(cuda, depth):
    rng = np.random.default_rng(depth)
    H, W, rps = 77, 150, 20
    img = rng.integers(0, 1 << depth, (H, W)).astype(np.uint16)
    parts, offs, cnts, pos = [np.full(40, 7, np.uint8)], [], [], 40
    for s in range(0, H, rps):
        blk = img[s:s + rps]
        b = blk.astype("<u2").tobytes() if depth == 16 else R.pack(blk, depth).tobytes()
        b = np.frombuffer(b, np.uint8)
        offs.append(pos); cnts.append(len(b)); parts.append(b); pos += len(b)
    f = np.concatenate(parts)
    kw = dict(compression=1, tiled=False, rows_per_strip=rps, bit_depth=depth)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)
