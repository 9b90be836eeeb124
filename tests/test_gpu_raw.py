"""PEF raw decoding on the GPU (isa_pef_decode, isa_pef_unpack) against the
restated reference decoder (oracle/raw.py), bit-exact: edge-case frames,
full-size frames of the benchmark's statistics, truncated and padded
streams, random streams through a partial code book (empty table entries,
which stop the reference's reader), and multi-strip uncompressed frames."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, synthetic

import raw as R

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_decode(stream, table, W, H):
    import torch
    out = isa.pef_decode(dev(stream), table, W, H)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint16)


BOOK = R.canonical_book()
TABLE = R.huff_table(R.maker_note_bytes(*BOOK))


@pytest.mark.parametrize("shape", [(1, 1), (1, 40), (23, 1), (8, 2), (3, 5), (37, 53), (64, 257), (300, 200)])
def test_decode_small_frames(cuda, shape):
    H, W = shape
    img = np.random.default_rng(H * 1000 + W).integers(0, 16384, shape).astype(np.uint16)
    s = R.encode(img, *BOOK)
    got = gpu_decode(s, TABLE, W, H)
    assert np.array_equal(got, img)
    assert np.array_equal(got, R.decode(s, TABLE, W, H))


def test_decode_full_frame(cuda):
    """A 6016 x 4000 frame of the benchmark burst, exact."""
    b = synthetic.make_burst(6016, 4000, 2, seed=77, max_shift=4, max_rot_deg=0.1)
    img = np.ascontiguousarray(b.raw[1])
    s = R.encode(img, *BOOK)
    got = gpu_decode(s, TABLE, 6016, 4000)
    assert np.array_equal(got, img)


@pytest.mark.parametrize("cut", [0.5, 0.9, 1.0, 1.3])
def test_decode_truncated_and_padded(cuda, cut):
    img = np.random.default_rng(5).integers(0, 16384, (120, 96)).astype(np.uint16)
    s = R.encode(img, *BOOK)
    n = int(len(s) * cut)
    t = s[:n] if cut <= 1 else np.concatenate([s, np.random.default_rng(6).integers(0, 256, n - len(s)).astype(np.uint8)])
    got = gpu_decode(t, TABLE, 96, 120)
    assert np.array_equal(got, R.decode(t, TABLE, 96, 120))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_decode_random_stream_partial_book(cuda, seed):
    """Random bytes through a book that leaves most 12-bit peeks empty: the
    reference's reader stops consuming at the first empty entry."""
    code, lens = R.canonical_book([3, 3, 4, 5, 6, 7, 8, 9, 10])
    mn = R.maker_note_bytes(code[:9], lens[:9])
    table = R.huff_table(mn)
    rng = np.random.default_rng(seed)
    s = rng.integers(0, 256, 4000 + 997 * seed).astype(np.uint8)
    W, H = 61, 47
    got = gpu_decode(s, table, W, H)
    assert np.array_equal(got, R.decode(s, table, W, H))


@pytest.mark.parametrize("depth,rows_per_strip", [(12, 1), (12, 7), (14, 16), (14, 3000), (16, 5), (10, 9)])
def test_unpack(cuda, depth, rows_per_strip):
    import torch
    rng = np.random.default_rng(depth + rows_per_strip)
    H, W = 301, 203
    img = rng.integers(0, 1 << depth, (H, W)).astype(np.uint16)
    packed = R.pack(img, depth)
    nstrips = (H + rows_per_strip - 1) // rows_per_strip
    head = 64  # strips start after a header, as in a file
    offs = [head + (s * rows_per_strip * W * depth + 7) // 8 for s in range(nstrips)]
    file = np.concatenate([np.full(head, 0x5A, np.uint8), packed])
    sizes = [len(file) - o for o in offs]
    out = isa.pef_unpack(dev(file), offs, sizes, rows_per_strip, W, H, depth)
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint16)
    assert np.array_equal(got, img)
    assert np.array_equal(got, R.unpack(file, offs, sizes, rows_per_strip, W, H, depth))
