"""PEF raw decoding without a GPU: the restated reference decoder
(oracle/raw.py over orc_pef_decode / orc_pef_unpack) inverts the stream
synthesiser on edge-case images, and the host entry points of libisa.so
(isa_pef_huff_table, isa_pef_levels) equal the restatement. There are no
PEF files or reference-produced decodes here, so the decoder's parity is
pinned only by these round trips (parity unpinned)."""
import ctypes

import numpy as np
import pytest

from imagestackalignator_b200 import isa

import raw as R


def images():
    rng = np.random.default_rng(1)
    yield "noise", np.clip(rng.normal(3000, 900, (37, 53)), 0, 16383).astype(np.uint16)
    yield "extremes", rng.choice([0, 16383], (16, 31)).astype(np.uint16)
    yield "flat", np.full((9, 12), 512, np.uint16)
    yield "one_row", rng.integers(0, 16384, (1, 40)).astype(np.uint16)
    yield "one_col", rng.integers(0, 16384, (23, 1)).astype(np.uint16)
    yield "two_cols", rng.integers(0, 16384, (8, 2)).astype(np.uint16)
    y, x = np.mgrid[0:64, 0:80]
    yield "smooth", (2000 + 800 * np.sin(x / 7.0) * np.cos(y / 11.0) + rng.normal(0, 20, (64, 80))).astype(np.uint16)


@pytest.mark.parametrize("name,img", list(images()), ids=[n for n, _ in images()])
@pytest.mark.parametrize("big_endian", [False, True])
def test_oracle_decode_inverts_encoder(name, img, big_endian):
    code, lens = R.canonical_book()
    table = R.huff_table(R.maker_note_bytes(code, lens, big_endian), big_endian)
    s = R.encode(img, code, lens)
    H, W = img.shape
    assert np.array_equal(R.decode(s, table, W, H), img)
    # trailing bytes after the strip do not change the frame
    assert np.array_equal(R.decode(np.concatenate([s, np.full(9, 0xA5, np.uint8)]), table, W, H), img)


def test_oracle_decode_reads_zeros_past_the_end():
    code, lens = R.canonical_book()
    table = R.huff_table(R.maker_note_bytes(code, lens))
    img = np.random.default_rng(2).integers(0, 16384, (10, 20)).astype(np.uint16)
    s = R.encode(img, code, lens)
    cut = R.decode(s[: len(s) // 2], table, 20, 10)
    padded = R.decode(np.concatenate([s[: len(s) // 2], np.zeros(len(s), np.uint8)]), table, 20, 10)
    assert np.array_equal(cut, padded)


@pytest.mark.parametrize("depth", [10, 12, 14, 16])
@pytest.mark.parametrize("rows_per_strip", [1, 7, 31])
def test_oracle_unpack(depth, rows_per_strip):
    rng = np.random.default_rng(depth * 100 + rows_per_strip)
    H, W = 31, 45
    img = rng.integers(0, 1 << depth, (H, W)).astype(np.uint16)
    packed = R.pack(img, depth)
    # strips laid out back to back in one buffer: strip s starts at the first byte it has not
    # consumed yet, so the reader's left-over bits continue the stream
    nstrips = (H + rows_per_strip - 1) // rows_per_strip
    offs = [(s * rows_per_strip * W * depth + 7) // 8 for s in range(nstrips)]
    sizes = [len(packed) - o for o in offs]
    pad = np.concatenate([packed, np.zeros(8, np.uint8)])
    assert np.array_equal(R.unpack(pad, offs, sizes, rows_per_strip, W, H, depth), img)


@pytest.mark.parametrize("big_endian", [False, True])
def test_huff_table_matches_oracle(big_endian):
    for lens in (R.DEFAULT_LENGTHS, [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 12]):
        code, ln = R.canonical_book(lens)
        mn = R.maker_note_bytes(code, ln, big_endian)
        assert np.array_equal(isa.pef_huff_table(mn, big_endian), R.huff_table(mn, big_endian))


@pytest.mark.parametrize("cfa,bp,wl", [([0, 1, 1, 2], [510, 512, 514, 516], 16383), ([1, 0, 2, 1], [500, 501, 502, 503], 16383),
                                       ([2, 1, 1, 0], [600], 4095), ([0, 1, 1, 2], [1, 2, 3], None), ([1, 2, 0, 1], None, None)])
def test_levels_match_oracle(cfa, bp, wl):
    got = isa.pef_levels(cfa, bp, wl, [100, 200, 300, 400], 256.0, 14)
    want = R.levels(cfa, bp, wl, [100, 200, 300, 400], 256.0, 14)
    for g, w in zip(got, want):
        assert np.array_equal(np.float32(g), np.float32(w))


def test_pef_argument_checks():
    lib = isa.lib()
    fake = ctypes.c_void_p(256)
    code, lens = R.canonical_book()
    t = R.huff_table(R.maker_note_bytes(code, lens))
    tp = t.ctypes.data_as(ctypes.c_void_p)
    need = lib.isa_pef_decode_scratch(ctypes.c_size_t(1000), 64, 32)
    assert need > 64 * 32 * 4
    args = lambda tab, scr: (fake, ctypes.c_size_t(1000), tab, 64, 32, fake, ctypes.c_size_t(scr), fake, ctypes.c_size_t(128), None)
    assert lib.isa_pef_decode(*args(tp, need - 1)) == isa.ISA_EINVAL
    bad = t.copy()
    bad[5] = (13 << 8) | 2       # code longer than the 12-bit peek
    assert lib.isa_pef_decode(*args(bad.ctypes.data_as(ctypes.c_void_p), need)) == isa.ISA_EINVAL
    bad = t.copy()
    bad[0] = 11
    assert lib.isa_pef_decode(*args(bad.ctypes.data_as(ctypes.c_void_p), need)) == isa.ISA_EINVAL
    off = np.zeros(1, np.uint32)
    sz = np.ones(1, np.uint32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.isa_pef_unpack(fake, ctypes.c_size_t(10), p(off), p(sz), 1, 4, 8, 8, 12, fake, ctypes.c_size_t(16), None) == isa.ISA_EINVAL
    assert lib.isa_pef_unpack(fake, ctypes.c_size_t(10), p(off), p(sz), 1, 8, 8, 8, 17, fake, ctypes.c_size_t(16), None) == isa.ISA_EINVAL
    assert lib.isa_pef_huff_table(p(np.zeros(4, np.uint8)), ctypes.c_size_t(4), 0, p(np.zeros(4097, np.uint16))) == isa.ISA_EINVAL


def test_synthesisers_match_the_oracle_encoders():
    """The numpy stream builders bench.py uses (imagestackalignator_b200/synthetic.py)
    write the same bytes as the oracle's encoders, which the restated readers invert."""
    from imagestackalignator_b200 import synthetic as S
    rng = np.random.default_rng(8)
    code, lens = S.pef_code_book()
    for shape in [(1, 1), (8, 2), (37, 53)]:
        img = rng.integers(0, 16384, shape).astype(np.uint16)
        assert np.array_equal(S.pef_stream(img, code, lens), R.encode(img, code, lens))
    for clrs in (1, 2):
        img = np.clip(rng.normal(3000, 700, (24, 32)), 0, 16383).astype(np.uint16)
        t = S.lj92_tile(img, clrs, 14)
        assert np.array_equal(t, R.lj92_encode(img, clrs, 14, 1, 0))
        st, out = R.dng_decode(np.concatenate([np.zeros(8, np.uint8), t]), 32, 24, [8], [len(t)], tiled=True, tile_w=32, tile_h=24)
        assert st == 0 and np.array_equal(out, img)


@pytest.mark.parametrize("psv", [1, 4, 7])
def test_oracle_dng_tiles_round_trip(psv):
    rng = np.random.default_rng(psv)
    img = np.clip(rng.normal(3000, 400, (50, 70)), 0, 16383).astype(np.uint16)
    f, offs, cnts = R.dng_tiles(img, 32, 32, clrs=2, bits=14, psv=psv)
    st, out = R.dng_decode(f, 70, 50, offs, cnts, tiled=True, tile_w=32, tile_h=32)
    assert st == 0 and np.array_equal(out, img)
