"""CPU restatement of the PEF raw decoding (test infrastructure: only tests/,
the smoke check and bench.py's CPU baseline use it), over oracle/isa_oracle.c:

  orc_pef_huff_table -- MNHuffmanTable (PefFile/PentaxMakerNotesEntry.cs:4555-4613)
  orc_pef_decode     -- PEFFile compressed branch (PefFile/PEFFile.cs:35-111)
  orc_pef_unpack     -- PEFFile uncompressed branch (PefFile/PEFFile.cs:116-156)
  orc_pef_encode     -- the inverse of the decoder, to synthesise test streams

plus the black/white/white-balance derivation of PEFFile.SetMembers
(PefFile/PEFFile.cs:176-280). There are no PEF files here: the tests build
streams and maker-note tables with the synthesiser below and check the GPU
decoder against the restated reference decoder on them.
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_L = None


def lib():
    global _L
    if _L is None:
        _L = ctypes.CDLL(os.path.join(HERE, "_build", "liboracle64.so"))
        _L.orc_pef_huff_table.restype = ctypes.c_int
        _L.orc_pef_encode.restype = ctypes.c_long
    return _L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# Code lengths per difference category 0..14 (a JPEG-like DC book extended to
# 14-bit differences); Kraft sum 0.9998 <= 1.
DEFAULT_LENGTHS = [2, 3, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12]


def canonical_book(lengths=DEFAULT_LENGTHS):
    """Canonical prefix code for the given lengths: code words left-aligned in 12 bits."""
    order = sorted(range(len(lengths)), key=lambda c: (lengths[c], c))
    code = [0] * len(lengths)
    nxt, prev = 0, lengths[order[0]]
    for i, c in enumerate(order):
        if i:
            nxt = (nxt + 1) << (lengths[c] - prev)
        prev = lengths[c]
        code[c] = nxt << (12 - lengths[c])
    assert all(code[c] >> (12 - lengths[c]) < (1 << lengths[c]) for c in range(len(lengths)))
    return np.array(code, np.uint16), np.array(lengths, np.uint8)


def maker_note_bytes(code, lens, big_endian=False):
    """The HuffmanTable maker-note payload MNHuffmanTable parses."""
    dep = len(code)
    e = ">" if big_endian else "<"
    return struct.pack(e + "H", (dep - 12) & 0xFFFF) + bytes(12) + struct.pack(e + f"{dep}H", *[int(c) for c in code]) + bytes(
        int(v) for v in lens)


def huff_table(mn, big_endian=False):
    t = np.zeros(4097, np.uint16)
    buf = np.frombuffer(bytes(mn), np.uint8).copy()
    dep = lib().orc_pef_huff_table(_p(buf), len(buf), int(big_endian), _p(t))
    if dep < 0:
        raise ValueError("short maker note")
    return t


def encode(img, code, lens):
    img = np.ascontiguousarray(img, np.uint16)
    H, W = img.shape
    cap = img.size * 4 + 16
    out = np.zeros(cap, np.uint8)
    n = lib().orc_pef_encode(_p(img), W, H, _p(np.ascontiguousarray(code, np.uint16)), _p(np.ascontiguousarray(lens, np.uint8)), len(code),
                             _p(out), ctypes.c_size_t(cap))
    if n < 0:
        raise ValueError("difference outside the code book")
    return out[:n].copy()


def decode(data, table, W, H):
    d = np.ascontiguousarray(data, np.uint8)
    out = np.zeros((H, W), np.uint16)
    lib().orc_pef_decode(_p(d), ctypes.c_size_t(d.size), _p(np.ascontiguousarray(table, np.uint16)), W, H, _p(out))
    return out


def unpack(file, offsets, sizes, rows_per_strip, W, H, depth):
    f = np.ascontiguousarray(file, np.uint8)
    off = np.ascontiguousarray(offsets, np.uint32)
    sz = np.ascontiguousarray(sizes, np.uint32)
    out = np.zeros((H, W), np.uint16)
    lib().orc_pef_unpack(_p(f), ctypes.c_size_t(f.size), _p(off), _p(sz), len(off), rows_per_strip, W, H, depth, _p(out))
    return out


def pack(img, depth):
    """MSB-first packing of W x H values of `depth` bits into one byte run (zero-padded)."""
    v = np.ascontiguousarray(img, np.uint64).reshape(-1)
    bits = ((v[:, None] >> np.arange(depth - 1, -1, -1, dtype=np.uint64)) & 1).astype(np.uint8).reshape(-1)
    return np.packbits(bits)


def levels(bayer, black_point, white_level, white_point, scaling, bit_depth):
    """PEFFile.SetMembers black / white / white balance (PEFFile.cs:199-260):
    returns (black[3], white[3] (white excludes black), wb[3])."""
    white_all = np.float32(2.0 ** bit_depth) if white_level is None else np.float32(white_level)
    black = [np.float32(0)] * 3
    if black_point is not None:
        bp = [np.float32(v) for v in black_point]
        if len(bp) == 1:
            black = [bp[0]] * 3
        elif len(bp) == 3:
            black = bp
        elif len(bp) == 4:
            r = [i for i, c in enumerate(bayer) if c == 0][0]
            b = [i for i, c in enumerate(bayer) if c == 2][0]
            g = [i for i, c in enumerate(bayer) if c == 1]
            black = [bp[r], max(bp[g[0]], bp[g[-1]]), bp[b]]
    white = [np.float32(white_all - black[c]) for c in range(3)]
    s = np.float32(scaling)
    wb = [np.float32(np.float32(white_point[0]) / s), np.float32(np.float32(white_point[1]) / s), np.float32(np.float32(white_point[3]) / s)]
    return black, white, wb


# ---- DNG (lossless JPEG tiles / strips, uncompressed strips) ----

def lj92_encode(img, clrs=1, bits=14, psv=1, restart=0, lens=(2, 3, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13)):
    """A lossless-JPEG tile (SOI, SOF3, DHT, DRI, SOS, data, EOI) of img (high x wide*clrs, interleaved components)."""
    img = np.ascontiguousarray(img, np.uint16)
    high, W = img.shape
    wide = W // clrs
    L = lib()
    L.orc_lj92_encode.restype = ctypes.c_long
    cap = img.size * 5 + 1024
    out = np.zeros(cap, np.uint8)
    ln = np.ascontiguousarray(lens, np.uint8)
    n = L.orc_lj92_encode(_p(img), wide, high, clrs, bits, psv, restart, _p(ln), len(ln), _p(out), ctypes.c_size_t(cap))
    if n < 0:
        raise ValueError("difference outside the code book")
    return out[:n].copy()


def dng_decode(file, W, H, offsets, counts, compression=7, tiled=True, tile_w=0, tile_h=0, rows_per_strip=0, bit_depth=16, large=True,
               linearization=None, black_h=None, black_v=None):
    """DNGFile pixel data of a file image (uint8): returns (status, uint16 H x W)."""
    f = np.ascontiguousarray(file, np.uint8)
    off = np.ascontiguousarray(offsets, np.uint32)
    cnt = np.ascontiguousarray(counts, np.uint32)
    lin = None if linearization is None else np.ascontiguousarray(linearization, np.uint16)
    bh = None if black_h is None else np.ascontiguousarray(black_h, np.uint16)
    bv = None if black_v is None else np.ascontiguousarray(black_v, np.uint16)
    out = np.zeros((H, W), np.uint16)
    L = lib()
    L.orc_dng_decode.restype = ctypes.c_int
    st = L.orc_dng_decode(_p(f), ctypes.c_size_t(f.size), int(tiled), tile_w, tile_h, rows_per_strip, len(off), _p(off), _p(cnt), compression,
                          bit_depth, int(large), None if lin is None else _p(lin), 0 if lin is None else lin.size,
                          None if bh is None else _p(bh), None if bv is None else _p(bv), W, H, _p(out))
    return st, out


def dng_tiles(img, tile_w, tile_h, clrs=1, bits=14, psv=1, restart=0, head=32):
    """A file image with the frame cut into lossless-JPEG tiles (tile_w pixels = tile_w / clrs samples of clrs components),
    tiles in row-major order after `head` bytes; returns (file, offsets, counts)."""
    H, W = img.shape
    parts = [np.full(head, 0x42, np.uint8)]
    offs, cnts = [], []
    pos = head
    for ty in range(0, H, tile_h):
        for tx in range(0, W, tile_w):
            t = np.zeros((tile_h, tile_w), np.uint16)
            blk = img[ty:ty + tile_h, tx:tx + tile_w]
            t[:blk.shape[0], :blk.shape[1]] = blk
            s = lj92_encode(t, clrs, bits, psv, restart)
            offs.append(pos)
            cnts.append(len(s))
            parts.append(s)
            pos += len(s)
    return np.concatenate(parts), offs, cnts
