"""Seeded synthetic Bayer bursts (the stand-in for real PEF/DNG bursts).

A linear-RGB scene is drawn from Gaussian blobs, straight and curved step
edges, sinusoidal gratings (period 2-16 px) and a checker patch. Each frame
is the scene under a global rotation about the frame centre and a translation
(frame 0 is the reference, unmoved), resampled with bicubic interpolation,
mosaicked with the CFA, given Poisson-Gaussian noise of variance a*x + b
(full scale) and quantised to unsigned 16-bit values with a black level.

The metadata follows the reference RawFile fields (PefFile/RawFile.cs:94-119):
WhiteLevel excludes the black level (PEFFile.cs:271-274, DNGFile.cs:832-834),
so values map to [0, 1] by (raw - black) / white.

Rendering uses torch (CPU or CUDA) only as a resampler for test data.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

CFA_CODES = {"RGGB": (0, 1, 1, 2), "BGGR": (2, 1, 1, 0), "GRBG": (1, 0, 2, 1), "GBRG": (1, 2, 0, 1)}


@dataclass
class Burst:
    raw: np.ndarray                  # n x H x W uint16
    cfa: tuple                       # codes at (0,0), (0,1), (1,0), (1,1)
    black: tuple                     # per R, G, B
    white: tuple                     # per R, G, B, black excluded
    noise_a: float
    noise_b: float
    shifts: np.ndarray               # n x 2 true translation (px) of each frame
    rotations: np.ndarray            # n true rotation (degrees)
    truth: Optional[np.ndarray] = None  # H x W x 3 clean linear scene of frame 0 (float64)
    camera_white: tuple = (1.0, 1.0, 1.0)
    meta: dict = field(default_factory=dict)
    object_path: Optional[np.ndarray] = None  # n x 2 centre (frame px) of the independently moving object, if any

    @property
    def n(self):
        return self.raw.shape[0]

    @property
    def height(self):
        return self.raw.shape[1]

    @property
    def width(self):
        return self.raw.shape[2]


def _render_scene(Wp, Hp, rng, torch, device, dtype):
    """Procedural linear-RGB scene on a Wp x Hp grid, values in about [0.03, 0.9].
    Each element is drawn inside its bounding box only."""
    yy = torch.arange(Hp, device=device, dtype=dtype).view(Hp, 1)
    xx = torch.arange(Wp, device=device, dtype=dtype).view(1, Wp)
    base = torch.tensor(rng.uniform(0.15, 0.45, 3), device=device, dtype=dtype)
    grad = torch.tensor(rng.uniform(-0.1, 0.1, (2, 3)), device=device, dtype=dtype)
    img = base.view(3, 1, 1) + grad[0].view(3, 1, 1) * (xx / Wp - 0.5) + grad[1].view(3, 1, 1) * (yy / Hp - 0.5)
    img = img.contiguous()
    area = Wp * Hp
    unit = max(1, int(area / (512 * 384)))
    scale = max(float(np.sqrt(area / (2048 * 1536))), 0.25)

    def color(lo=-0.25, hi=0.25):
        return torch.tensor(rng.uniform(lo, hi, 3), device=device, dtype=dtype).view(3, 1, 1)

    def box(cx, cy, r):
        x0, x1 = max(int(cx - r), 0), min(int(cx + r) + 1, Wp)
        y0, y1 = max(int(cy - r), 0), min(int(cy + r) + 1, Hp)
        return x0, x1, y0, y1

    def add(cx, cy, r, fn):
        x0, x1, y0, y1 = box(cx, cy, r)
        if x1 <= x0 or y1 <= y0:
            return
        X, Y = xx[:, x0:x1], yy[y0:y1, :]
        img[:, y0:y1, x0:x1] += fn(X, Y)

    for _ in range(24 * unit):  # Gaussian blobs
        cx, cy = rng.uniform(0, Wp), rng.uniform(0, Hp)
        s = rng.uniform(4, 60) * min(scale, 1.0)
        c = color()
        add(cx, cy, 4 * s, lambda X, Y: c * torch.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s)))
    for _ in range(8 * unit):  # straight step edges inside a window
        cx, cy = rng.uniform(0, Wp), rng.uniform(0, Hp)
        th = rng.uniform(0, np.pi)
        hw = rng.uniform(20, 160) * min(scale, 1.0)
        c = color()
        add(cx, cy, hw, lambda X, Y: c * (((X - cx) * np.cos(th) + (Y - cy) * np.sin(th)) > 0).to(dtype))
    for _ in range(8 * unit):  # curved edges: discs
        cx, cy = rng.uniform(0, Wp), rng.uniform(0, Hp)
        r = rng.uniform(10, 120) * min(scale, 1.0)
        c = color()
        add(cx, cy, r + 1, lambda X, Y: c * (((X - cx) ** 2 + (Y - cy) ** 2) < r * r).to(dtype))
    for _ in range(6 * unit):  # sinusoidal gratings, period 2..16 px
        cx, cy = rng.uniform(0, Wp), rng.uniform(0, Hp)
        period = rng.uniform(2, 16)
        th = rng.uniform(0, np.pi)
        hw = rng.uniform(20, 120) * min(scale, 1.0)
        c = color(0.05, 0.2)
        add(cx, cy, hw, lambda X, Y: c * torch.sin(2 * np.pi / period * ((X - cx) * np.cos(th) + (Y - cy) * np.sin(th))))
    for _ in range(max(1, unit // 8)):  # checker patches
        cx, cy = rng.uniform(0.1, 0.9) * Wp, rng.uniform(0.1, 0.9) * Hp
        sq = int(rng.integers(4, 17))
        c = color(0.1, 0.2)
        add(cx, cy, 80, lambda X, Y: c * (((torch.floor(X / sq) + torch.floor(Y / sq)) % 2) * 2 - 1))
    return img.clamp(0.03, 0.9)


def make_burst(width=2048, height=1536, frames=8, seed=0, max_shift=6.0, max_rot_deg=0.2,
               noise_a=4e-4, noise_b=2e-6, black=512, white_max=16383, cfa="RGGB", device="cpu",
               keep_truth=False, dtype=None, moving_object=0.0, object_step=(2.0, 40.0)) -> Burst:
    """Seeded burst; frame 0 is the reference with zero motion.

    moving_object > 0 adds a rigid textured disc covering that fraction of
    the frame area, which moves independently of the camera: each frame it
    steps object_step[0]..object_step[1] px in a random direction (reflected
    at the frame edges), occluding the background."""
    import torch
    import torch.nn.functional as F

    if dtype is None:
        dtype = torch.float64 if device == "cpu" else torch.float32
    rng = np.random.default_rng(seed)
    margin = int(np.ceil(max_shift + np.deg2rad(max_rot_deg) * 0.5 * np.hypot(width, height))) + 4
    Wp, Hp = width + 2 * margin, height + 2 * margin
    scene = _render_scene(Wp, Hp, rng, torch, device, dtype)
    shifts = np.zeros((frames, 2))
    rots = np.zeros(frames)
    shifts[1:] = rng.uniform(-max_shift, max_shift, (frames - 1, 2))
    rots[1:] = rng.uniform(-max_rot_deg, max_rot_deg, frames - 1)
    codes = CFA_CODES[cfa]
    ys, xs = torch.meshgrid(torch.arange(height, device=device, dtype=dtype),
                            torch.arange(width, device=device, dtype=dtype), indexing="ij")
    cfa_idx = ((ys.long() & 1) * 2 + (xs.long() & 1))
    chan = torch.tensor(codes, device=device)[cfa_idx]
    raw = np.empty((frames, height, width), dtype=np.uint16)
    gen = torch.Generator(device=device).manual_seed(int(seed) * 7919 + 17)
    truth = None
    obj = None
    if moving_object > 0:
        orng = np.random.default_rng(int(seed) * 104729 + 7)
        rad = float(np.sqrt(moving_object * width * height / np.pi))
        side = int(np.ceil(2 * rad)) + 8
        tex = _render_scene(side, side, orng, torch, device, dtype)
        pos = np.zeros((frames, 2))
        lo = np.array([rad + 2, rad + 2])
        hi = np.array([width - rad - 3, height - rad - 3])
        pos[0] = orng.uniform(lo, hi)
        for f in range(1, frames):
            ang = orng.uniform(0, 2 * np.pi)
            step = orng.uniform(*object_step)
            p = pos[f - 1] + step * np.array([np.cos(ang), np.sin(ang)])
            p = np.where(p < lo, 2 * lo - p, p)
            p = np.where(p > hi, 2 * hi - p, p)
            pos[f] = np.clip(p, lo, hi)
        obj = (tex, rad, side, pos)
    for f in range(frames):
        th = np.deg2rad(rots[f])
        c, s = np.cos(th), np.sin(th)
        cxf, cyf = (width - 1) / 2.0, (height - 1) / 2.0
        # frame pixel p sees scene point R(th) (p - c) + c + t
        dx, dy = xs - cxf, ys - cyf
        sx = c * dx - s * dy + cxf + shifts[f, 0] + margin
        sy = s * dx + c * dy + cyf + shifts[f, 1] + margin
        grid = torch.stack([(sx + 0.5) / Wp * 2 - 1, (sy + 0.5) / Hp * 2 - 1], dim=-1)[None]
        frame = F.grid_sample(scene[None], grid, mode="bicubic", padding_mode="border", align_corners=False)[0]
        if obj is not None:
            tex, rad, side, pos = obj
            ox, oy = xs - pos[f, 0] + side / 2.0, ys - pos[f, 1] + side / 2.0
            inside = ((xs - pos[f, 0]) ** 2 + (ys - pos[f, 1]) ** 2) <= rad * rad
            og = torch.stack([(ox + 0.5) / side * 2 - 1, (oy + 0.5) / side * 2 - 1], dim=-1)[None]
            ocol = F.grid_sample(tex[None], og, mode="bilinear", padding_mode="border", align_corners=False)[0]
            frame = torch.where(inside[None], ocol, frame)
            del og, ocol, inside
        frame = frame.clamp(0, 1)
        if f == 0 and keep_truth:
            truth = frame.permute(1, 2, 0).double().cpu().numpy()
        mosaic = torch.gather(frame, 0, chan[None]).squeeze(0)
        noise = torch.randn(mosaic.shape, generator=gen, device=device, dtype=dtype)
        noisy = mosaic + torch.sqrt(noise_a * mosaic + noise_b) * noise
        q = torch.round(black + noisy * (white_max - black)).clamp(0, white_max)
        raw[f] = q.to(torch.int32).cpu().numpy().astype(np.uint16)
        del frame, mosaic, noise, noisy, q, grid
    w = float(white_max - black)
    return Burst(raw=raw, cfa=codes, black=(float(black),) * 3, white=(w, w, w), noise_a=noise_a, noise_b=noise_b,
                 shifts=shifts, rotations=rots, truth=truth, object_path=None if obj is None else obj[3])


# ---- PEF-style compressed streams (inputs for isa_pef_decode) ----
# The reference only decodes; these build streams in the layout its decoder
# reads (PefFile/PEFFile.cs:81-111): per pixel in raster order a prefix code
# for the difference category (bit length of |diff|), then the difference in
# that many bits (negative values as diff - 1), the difference taken to the
# pixel two columns left, or two rows up in the first two columns.

PEF_CODE_LENGTHS = (2, 3, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12)


def pef_code_book(lengths=PEF_CODE_LENGTHS):
    """Canonical prefix code for the category lengths: (code words left-aligned in 12 bits, lengths)."""
    order = sorted(range(len(lengths)), key=lambda c: (lengths[c], c))
    code = [0] * len(lengths)
    nxt, prev = 0, lengths[order[0]]
    for i, c in enumerate(order):
        if i:
            nxt = (nxt + 1) << (lengths[c] - prev)
        prev = lengths[c]
        code[c] = nxt << (12 - lengths[c])
    return np.array(code, np.uint16), np.array(lengths, np.uint8)


def pef_maker_note(code, lens, big_endian=False):
    """The HuffmanTable maker-note payload (PefFile/PentaxMakerNotesEntry.cs:4555-4613)."""
    import struct
    e = ">" if big_endian else "<"
    dep = len(code)
    return (struct.pack(e + "H", (dep - 12) & 0xFFFF) + bytes(12) + struct.pack(e + f"{dep}H", *[int(c) for c in code]) +
            bytes(int(v) for v in lens))


def pef_stream(img, code, lens):
    """Compressed stream of a uint16 H x W frame (numpy, vectorised)."""
    v = np.asarray(img, np.int64)
    H, W = v.shape
    d = np.empty_like(v)
    d[:, 2:] = v[:, 2:] - v[:, :-2]
    d[:2, :2] = v[:2, :2]
    d[2:, :2] = v[2:, :2] - v[:-2, :2]
    d = d.reshape(-1)
    mag = np.abs(d)
    ssss = np.zeros(mag.shape, np.int64)
    while True:
        m = (mag >> ssss) != 0
        if not m.any():
            break
        ssss += m
    if ssss.max() >= len(code):
        raise ValueError("difference outside the code book")
    clen = np.asarray(lens, np.int64)[ssss]
    cword = np.asarray(code, np.int64)[ssss] >> (12 - clen)
    dbits = np.where(d >= 0, d, d - 1) & ((np.int64(1) << ssss) - 1)
    field = (cword << ssss) | dbits          # code then difference, MSB first
    flen = clen + ssss
    start = np.concatenate([[0], np.cumsum(flen)[:-1]])
    total = int(start[-1] + flen[-1])
    # each field (at most 26 bits) lies in the 64-bit big-endian pair of 32-bit words (w, w + 1)
    w = start >> 5
    val = (field << (64 - (start & 31) - flen)).astype(np.uint64)
    hi = val >> np.uint64(32)
    lo = val & np.uint64(0xFFFFFFFF)
    words = np.zeros(int(w[-1]) + 2, np.uint64)
    first = np.concatenate([[0], np.flatnonzero(np.diff(w)) + 1])
    words[w[first]] |= np.bitwise_or.reduceat(hi, first)
    words[w[first] + 1] |= np.bitwise_or.reduceat(lo, first)
    return np.frombuffer(words.astype(">u4").tobytes(), np.uint8)[: (total + 7) // 8].copy()


# ---- Lossless-JPEG (DNG) tiles, inputs for isa_dng_decode ----

LJ92_CODE_LENGTHS = (2, 3, 3, 3, 3, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13)


def _bits_to_bytes(field, flen):
    """Concatenate MSB-first bit fields (each at most 26 bits) into bytes, the last one padded with ones."""
    field = np.asarray(field, np.int64)
    flen = np.asarray(flen, np.int64)
    start = np.concatenate([[0], np.cumsum(flen)[:-1]])
    total = int(start[-1] + flen[-1]) if len(flen) else 0
    pad = (-total) % 8
    if pad:
        field = np.concatenate([field, [(1 << pad) - 1]])
        flen = np.concatenate([flen, [pad]])
        start = np.concatenate([start, [total]])
        total += pad
    w = start >> 5
    val = (field << (64 - (start & 31) - flen)).astype(np.uint64)
    hi = val >> np.uint64(32)
    lo = val & np.uint64(0xFFFFFFFF)
    words = np.zeros(int(w[-1]) + 2, np.uint64)
    first = np.concatenate([[0], np.flatnonzero(np.diff(w)) + 1])
    words[w[first]] |= np.bitwise_or.reduceat(hi, first)
    words[w[first] + 1] |= np.bitwise_or.reduceat(lo, first)
    return np.frombuffer(words.astype(">u4").tobytes(), np.uint8)[: total // 8].copy()


def lj92_tile(img, clrs=2, bits=14, lengths=LJ92_CODE_LENGTHS):
    """One lossless-JPEG tile (predictor 1, one Huffman table for all
    components, no restart interval) of a uint16 high x (wide * clrs) block
    whose components are interleaved, in the layout DNGFile's reader
    (PefFile/DNGFile.cs:94-285) decodes."""
    v = np.asarray(img, np.int64)
    high, W = v.shape
    wide = W // clrs
    pred = np.empty_like(v)
    pred[:, clrs:] = v[:, :-clrs]                       # left sample of the same component
    pred[0, :clrs] = 1 << (bits - 1)                     # vpred at the first row
    pred[1:, :clrs] = v[:-1, :clrs]                      # the first column from the row above
    d = (v - pred) & 0xFFFF
    d = np.where(d >= 32768, d - 65536, d).reshape(-1)
    mag = np.abs(d)
    ssss = np.zeros(mag.shape, np.int64)
    while True:
        m = (mag >> ssss) != 0
        if not m.any():
            break
        ssss += m
    lens = np.asarray(lengths, np.int64)
    if ssss.max() >= len(lens):
        raise ValueError("difference outside the code book")
    code = np.zeros(len(lens), np.int64)
    c = 0
    for ln in range(1, 17):
        for k in range(len(lens)):
            if lens[k] == ln:
                code[k] = c
                c += 1
        c <<= 1
    clen = lens[ssss]
    dbits = np.where(d >= 0, d, d - 1) & ((np.int64(1) << ssss) - 1)
    data = _bits_to_bytes((code[ssss] << ssss) | dbits, clen + ssss)
    stuffed = np.insert(data, np.flatnonzero(data == 0xFF) + 1, 0)   # a zero byte after every 0xFF
    counts = [int((lens == ln).sum()) for ln in range(1, 17)]
    values = [k for ln in range(1, 17) for k in range(len(lens)) if lens[k] == ln]
    hdr = bytearray([0xFF, 0xD8, 0xFF, 0xC3, 0, 8 + 3 * clrs, bits, high >> 8, high & 255, wide >> 8, wide & 255, clrs])
    for c in range(clrs):
        hdr += bytes([c + 1, 0x11, 0])
    hdr += bytes([0xFF, 0xC4, 0, 3 + 16 + len(values), 0x00]) + bytes(counts) + bytes(values)
    hdr += bytes([0xFF, 0xDA, 0, 6 + 2 * clrs, clrs])
    for c in range(clrs):
        hdr += bytes([c + 1, 0x00])
    hdr += bytes([1, 0, 0])
    return np.concatenate([np.frombuffer(bytes(hdr), np.uint8), stuffed, np.array([0xFF, 0xD9], np.uint8)])


def dng_tiled_file(img, tile_w=256, tile_h=256, clrs=2, bits=14, head=64):
    """A file image holding `img` as lossless-JPEG tiles in row-major order
    after `head` bytes: (file, offsets, byte counts)."""
    H, W = img.shape
    parts = [np.zeros(head, np.uint8)]
    offs, cnts, pos = [], [], head
    for ty in range(0, H, tile_h):
        for tx in range(0, W, tile_w):
            t = np.zeros((tile_h, tile_w), np.uint16)
            blk = img[ty:ty + tile_h, tx:tx + tile_w]
            t[: blk.shape[0], : blk.shape[1]] = blk
            s = lj92_tile(t, clrs, bits)
            offs.append(pos)
            cnts.append(len(s))
            parts.append(s)
            pos += len(s)
    return np.concatenate(parts), offs, cnts


# ---- DNG files (TIFF container) ----

_TIFF_FMT = {1: "B", 3: "H", 4: "I", 5: "II", 7: "B", 10: "ii", 12: "d"}


def _ifd_bytes(entries, at, big, next_off):
    """One IFD written at file offset `at`: entries (tag, type, values) sorted by
    tag; values over 4 bytes follow the entry table."""
    import struct
    e = ">" if big else "<"
    entries = sorted(entries, key=lambda x: x[0])
    table_len = 2 + 12 * len(entries) + 4
    table = struct.pack(e + "H", len(entries))
    extra = b""
    for tag, typ, vals in entries:
        fmt = _TIFF_FMT[typ]
        flat = [v for pair in vals for v in pair] if typ in (5, 10) else list(vals)
        data = struct.pack(e + fmt[0] * len(flat), *flat)
        if len(data) <= 4:
            field = data + b"\0" * (4 - len(data))
        else:
            field = struct.pack(e + "I", at + table_len + len(extra))
            extra += data + (b"\0" if len(data) % 2 else b"")
        table += struct.pack(e + "HHI", tag, typ, len(vals)) + field
    table += struct.pack(e + "I", next_off)
    return table + extra


def _rat(v, den=1000):
    return (int(round(v * den)), den)


def dng_file(img, cfa=(0, 1, 1, 2), bits=14, tile=128, clrs=2, big_endian=False, raw_in_subifd=True, black=(512,), white=16383,
             active_area=None, crop=None, deltas=None, noise=None, plane_color=None, iso=200, color=None, version=(1, 4, 0, 0),
             linearization=None, extra_chain_ifd=False, private_note=None, roll_byte=0, threads=1):
    """A DNG file image holding `img` (uint16 H x W Bayer) as lossless-JPEG
    tiles in a CFA IFD (a SubIFD of IFD 0, or IFD 0 itself), with the tags
    DNGFile and DNGColorSpec read. color: dict of color_matrix1/2 (9 values),
    illuminant1/2, forward_matrix1, camera_calibration1, analog_balance,
    as_shot_neutral, as_shot_white_xy. Rationals are written with
    denominator 1000 (10000 for matrices)."""
    import struct
    H, W = img.shape
    e = ">" if big_endian else "<"
    out = bytearray((b"MM" if big_endian else b"II") + struct.pack(e + "HI", 42, 0))
    offs, cnts = [], []

    def encode(pos):
        ty, tx = pos
        t = np.zeros((tile, tile), np.uint16)
        blk = img[ty:ty + tile, tx:tx + tile]
        t[:blk.shape[0], :blk.shape[1]] = blk
        return lj92_tile(t, clrs, bits)

    positions = [(ty, tx) for ty in range(0, H, tile) for tx in range(0, W, tile)]
    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:
            tiles = list(ex.map(encode, positions))
    else:
        tiles = [encode(p) for p in positions]
    for s in tiles:
        offs.append(len(out))
        cnts.append(len(s))
        out += bytes(s)
        if len(out) % 2:
            out += b"\0"
    raw = [(254, 4, [0]), (256, 4, [W]), (257, 4, [H]), (258, 3, [16]), (259, 3, [7]), (262, 3, [32803]), (277, 3, [1]),
           (322, 3, [tile]), (323, 3, [tile]), (324, 4, offs), (325, 4, cnts), (33421, 3, [2, 2]), (33422, 1, list(cfa)),
           (50717, 4, [white])]
    if black is not None:
        raw.append((50714, 5, [_rat(b) for b in black]))
    if active_area is not None:
        raw.append((50829, 4, list(active_area)))
    if crop is not None:
        raw.append((50719, 5, [_rat(crop[0]), _rat(crop[1])]))
        raw.append((50720, 5, [_rat(crop[2]), _rat(crop[3])]))
    if deltas is not None:
        raw.append((50715, 10, [_rat(v) for v in deltas[0]]))
        raw.append((50716, 10, [_rat(v) for v in deltas[1]]))
    if noise is not None:
        raw.append((51041, 12, list(noise)))
    if plane_color is not None:
        raw.append((50710, 1, list(plane_color)))
    if linearization is not None:
        raw.append((50712, 3, [int(v) for v in linearization]))
    ifd0 = [(254, 4, [1]), (256, 4, [16]), (257, 4, [16]), (271, 2, [0]), (50706, 1, list(version))] if version else [(254, 4, [1])]
    ifd0 = [x for x in ifd0 if x[0] != 271]
    c = dict(color or {})
    for k, tag in (("color_matrix1", 50721), ("color_matrix2", 50722), ("forward_matrix1", 50964), ("forward_matrix2", 50965),
                   ("camera_calibration1", 50723)):
        if c.get(k) is not None:
            ifd0.append((tag, 10, [_rat(v, 10000) for v in c[k]]))
    for k, tag in (("illuminant1", 50778), ("illuminant2", 50779)):
        if c.get(k):
            ifd0.append((tag, 3, [int(c[k])]))
    for k, tag in (("analog_balance", 50727), ("as_shot_neutral", 50728), ("as_shot_white_xy", 50729)):
        if c.get(k) is not None:
            ifd0.append((tag, 5, [_rat(v, 10000) for v in c[k]]))
    if private_note is not None:
        # DNGPrivateData: "Adobe\0MakN", count, byte order, the note's original file offset, then a Pentax
        # maker note ("AOC": offsets from the original file's start; "PENTAX": from the note's start)
        orig = 123456
        level = [(0x022b, 1, [1, roll_byte & 0xFF, 0, 0, 0, 0, 0, 0, 0, 0]), (0x0201, 3, [8192, 8192, 8192, 8192])]
        if private_note == "AOC":
            head = b"AOC\0" + (b"MM" if big_endian else b"II")
            note_bytes = head + _ifd_bytes(level, orig + len(head), big_endian, 0)
        else:
            head = b"PENTAX \0" + (b"MM" if big_endian else b"II")
            note_bytes = head + _ifd_bytes(level, len(head), big_endian, 0)
        pdata = b"Adobe\0MakN" + struct.pack(">I", len(note_bytes) + 6) + (b"MM" if big_endian else b"II") + struct.pack(e + "I", orig) + note_bytes
        ifd0.append((50740, 1, list(pdata)))
    # the Exif IFD with the ISO, then the raw IFD, then IFD 0 (and a trailing chain IFD)
    exif_at = len(out)
    out += _ifd_bytes([(34855, 3, [iso])], exif_at, big_endian, 0)
    ifd0.append((34665, 4, [exif_at]))
    tail_at = 0
    if extra_chain_ifd:
        tail_at = len(out)
        out += _ifd_bytes([(254, 4, [1]), (256, 4, [8]), (257, 4, [8]), (262, 3, [2])], tail_at, big_endian, 0)
    if raw_in_subifd:
        raw_at = len(out)
        out += _ifd_bytes(raw, raw_at, big_endian, 0)
        ifd0.append((330, 4, [raw_at]))
        ifd0.append((262, 3, [2]))
        entries0 = ifd0
    else:
        entries0 = [x for x in ifd0 if x[0] not in (254, 256, 257)] + raw
    ifd0_at = len(out)
    out += _ifd_bytes(entries0, ifd0_at, big_endian, tail_at)
    struct.pack_into(e + "I", out, 4, ifd0_at)
    return np.frombuffer(bytes(out), np.uint8).copy(), offs, cnts


def pef_file(img, cfa=(0, 1, 1, 2), compressed=True, big_endian=False, note="AOC", note_big_endian=None, black=(512, 512, 512, 512),
             white_point=(8192, 8192, 8192, 8192), scaling=8192, white_level=16383, iso=400, bits=14, rows_per_strip=None, roll_byte=None):
    """A PEF file image holding `img` (uint16 H x W Bayer): IFD 0 with the
    strip(s), its Exif IFD with ISO, CFA pattern and a Pentax maker note
    ("AOC": entry offsets from the file's start, or "PENTAX": from the
    note's start) holding HuffmanTable (compressed frames), BlackPoint,
    WhitePoint, WhiteLevel and DataScaling. Uncompressed frames are stored
    as MSB-first `bits`-bit samples in strips of rows_per_strip rows."""
    import struct
    H, W = img.shape
    e = ">" if big_endian else "<"
    nb = big_endian if note_big_endian is None else note_big_endian
    out = bytearray((b"MM" if big_endian else b"II") + struct.pack(e + "HI", 42, 0))
    code, lens = pef_code_book()
    offs, cnts = [], []
    if compressed:
        data = pef_stream(img, code, lens)
        offs.append(len(out))
        cnts.append(len(data))
        out += bytes(data)
        rps = H
    else:
        rps = rows_per_strip or H
        for y in range(0, H, rps):
            blk = np.asarray(img[y:y + rps], np.uint64).reshape(-1)
            bitsarr = ((blk[:, None] >> np.arange(bits - 1, -1, -1, dtype=np.uint64)) & 1).astype(np.uint8).reshape(-1)
            data = np.packbits(bitsarr)
            offs.append(len(out))
            cnts.append(len(data))
            out += bytes(data)
    if len(out) % 2:
        out += b"\0"
    entries = []
    if compressed:
        entries.append((0x0220, 7, list(pef_maker_note(code, lens, nb))))
    if black is not None:
        entries.append((0x0200, 3, list(black)))
    entries += [(0x0201, 3, list(white_point)), (0x003d, 3, [scaling])]
    if white_level is not None:
        entries.append((0x007e, 4, [white_level]))
    if roll_byte is not None:   # LevelInfo: orientation, roll (-2 x degrees), pitch, ...
        entries.append((0x022b, 1, [1, roll_byte & 0xFF, 0, 0, 0, 0, 0, 0, 0, 0]))
    mn_at = len(out)
    if note == "AOC":
        head = b"AOC\0" + (b"MM" if nb else b"II")
        body = _ifd_bytes(entries, mn_at + len(head), nb, 0)   # offsets from the file's start
    else:
        head = b"PENTAX \0" + (b"MM" if nb else b"II")
        body = _ifd_bytes(entries, len(head), nb, 0)            # offsets from the note's start
    note_bytes = head + body
    out += note_bytes
    if len(out) % 2:
        out += b"\0"
    exif_at = len(out)
    exif = [(34855, 3, [iso]), (41730, 7, [0, 2, 0, 2] + list(cfa)), (37500, 7, list(note_bytes))]
    # the maker note's bytes are already in the file: point the MakerNote entry at them
    exif_bytes = bytearray(_ifd_bytes(exif, exif_at, big_endian, 0))
    n = struct.unpack_from(e + "H", exif_bytes, 0)[0]
    for i in range(n):
        tag = struct.unpack_from(e + "H", exif_bytes, 2 + 12 * i)[0]
        if tag == 37500:
            struct.pack_into(e + "I", exif_bytes, 2 + 12 * i + 8, mn_at)
    out += exif_bytes
    ifd0_at = len(out)
    ifd0 = [(254, 4, [0]), (256, 4, [W]), (257, 4, [H]), (258, 3, [bits]), (259, 3, [65535 if compressed else 1]), (262, 3, [32803]),
            (273, 4, offs), (278, 4, [rps]), (279, 4, cnts), (34665, 4, [exif_at])]
    out += _ifd_bytes(ifd0, ifd0_at, big_endian, 0)
    struct.pack_into(e + "I", out, 4, ifd0_at)
    return np.frombuffer(bytes(out), np.uint8).copy(), offs, cnts
