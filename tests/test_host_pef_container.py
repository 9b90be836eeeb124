"""The PEF container reader (isa_pef_open / isa_pef_file_info, host code of
libisa.so) without a GPU: files written by synthetic.pef_file in both byte
orders, with "AOC" and "PENTAX" maker notes (the maker note's byte order
independent of the file's), compressed and multi-strip uncompressed; the
parsed Huffman table, levels and strips through the oracle's restated
PEFFile decoder; files the reference cannot read."""
import struct

import numpy as np
import pytest

from imagestackalignator_b200 import isa, synthetic as S

import raw as R


def _img(h=48, w=80, seed=0):
    return np.random.default_rng(seed).integers(512, 16000, (h, w)).astype(np.uint16)


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("note", ["AOC", "PENTAX"])
@pytest.mark.parametrize("note_big", [False, True])
def test_compressed_file_reads_back(big, note, note_big):
    img = _img(seed=int(big) + 2 * int(note_big))
    f, offs, cnts = S.pef_file(img, cfa=(1, 2, 0, 1), big_endian=big, note=note, note_big_endian=note_big, black=(510, 512, 514, 516),
                               white_point=(9000, 8192, 8192, 11000), scaling=8192, white_level=16000, iso=1600)
    d = isa.pef_open(f)
    assert (d["width"], d["height"], d["bit_depth"], d["cfa"], d["iso"]) == (80, 48, 14, [1, 2, 0, 1], 1600)
    assert d["compressed"] and d["nstrips"] == 1 and d["strip_offsets"] == offs and d["strip_sizes"] == cnts
    assert d["huffman_big_endian"] == note_big
    code, lens = S.pef_code_book()
    assert d["huffman_table"] == S.pef_maker_note(code, lens, note_big)
    table = isa.pef_huff_table(d["huffman_table"], big_endian=d["huffman_big_endian"])
    assert np.array_equal(table, R.huff_table(d["huffman_table"], big_endian=note_big))
    o, n = offs[0], cnts[0]
    assert np.array_equal(R.decode(f[o:o + n], table, 80, 48), img)
    got = isa.pef_levels(d["cfa"], d["black_point"], d["white_level"], d["white_point"], d["scaling"], d["bit_depth"])
    want = R.levels(d["cfa"], d["black_point"], d["white_level"], d["white_point"], d["scaling"], d["bit_depth"])
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g, np.float32), np.asarray(w, np.float32))


def test_uncompressed_strips_read_back():
    img = _img(50, 64, seed=5) & 0x3FFF
    f, offs, cnts = S.pef_file(img, compressed=False, rows_per_strip=16, white_level=None, black=None)
    d = isa.pef_open(f)
    assert not d["compressed"] and d["huffman_table"] is None and d["nstrips"] == 4 and d["rows_per_strip"] == 16
    assert d["white_level"] is None and d["black_point"] is None
    assert np.array_equal(R.unpack(f, d["strip_offsets"], d["strip_sizes"], 16, 64, 50, 14), img)


@pytest.mark.parametrize("damage", ["no_exif", "note_header", "no_white_point", "cfa_3x2", "note_order"])
def test_unreadable_files(damage):
    img = _img(16, 16)
    f, offs, cnts = S.pef_file(img)
    b = bytearray(f.tobytes())
    if damage == "no_exif":
        i = bytes(b).find(struct.pack("<HHI", 34665, 4, 1))
        struct.pack_into("<H", b, i, 34666)
    elif damage == "note_header":
        i = bytes(b).find(b"AOC\0")
        b[i:i + 4] = b"XYZ\0"
    elif damage == "no_white_point":
        i = bytes(b).find(struct.pack("<HHI", 0x0201, 3, 4))
        struct.pack_into("<H", b, i, 0x0202)
    elif damage == "cfa_3x2":
        i = bytes(b).find(bytes([0, 2, 0, 2, 0, 1, 1, 2]))
        b[i + 1] = 3
    elif damage == "note_order":
        i = bytes(b).find(b"AOC\0")
        b[i + 4:i + 6] = b"IM"
    with pytest.raises(isa.IsaError) as e:
        isa.pef_open(bytes(b))
    assert e.value.code == isa.ISA_EINVAL


@pytest.mark.parametrize("note", ["AOC", "PENTAX"])
@pytest.mark.parametrize("roll_byte", [None, 0, 7, -12])
def test_roll_angle_from_level_info(note, roll_byte):
    """MNLevelInfo: the roll angle is -(signed byte 1) / 2 degrees; absent without the entry."""
    f, _, _ = S.pef_file(_img(16, 16), note=note, roll_byte=roll_byte, big_endian=note == "PENTAX")
    got = isa.pef_open(f)["roll_angle"]
    assert got == (None if roll_byte is None else -roll_byte / 2.0)
