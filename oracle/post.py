"""CPU restatement of the colour/tone post-processing and the 16-bit TIFF
writer (test infrastructure: only tests/ and bench.py's CPU baseline use it).

Follows ImageStackAlignatorController.SaveAs16BitTiff
(PEFStudioDX/ImageStackAlignatorController.cs:2197-2260) and
ProcessColorsAndShow (:2262-2320):

  ThresholdLTGT [0, CameraWhite] -> ColorTwist camera->ProPhoto ->
  ThresholdLTGT [0, 1] -> LUTCubic -> ColorTwist ProPhoto->sRGB(D50) ->
  Mul 2^Exposure -> GammasRGB (Kernels/kernel.cu:290-332) -> Mul 65535 | 255 ->
  ROI -> Convert (round to nearest even, saturate)

in float32 with every operation rounded on its own, the colour matrices in
float64 as DNGColorSpace (PefFile/DNGColorSpace.cs:36-65), DNGMatrix
(PefFile/DNGMatrix.cs:181-193, 232-254, 440-486) and DNGxyCoord
(PefFile/DNGxyCoord.cs:79-101, 175-181, 211-214), and the TIFF layout of
ImageFileDirectory(width, height).SaveAsTiff (PefFile/ImageFileDirectory.cs:75-123)
with the entry writers of PefFile/ImageFileDirectoryEntry.cs.

Parity: the gamma step is pinned against the reference's own GammasRGB
compiled for the host (oracle/_ref). NPP's ThresholdLTGT, ColorTwist, MulC
and Convert are restated from their documented definitions. NPP's LUTCubic
does not publish its polynomial: it is restated as the cubic through the
four nearest levels (per-segment coefficients in float64, Horner's rule in
float32), so that step is parity unpinned.
"""
from __future__ import annotations

import struct

import numpy as np

f32 = np.float32

PROPHOTO = [[0.7976749, 0.1351917, 0.0313534], [0.2880402, 0.7118741, 0.0000857], [0.0000000, 0.0000000, 0.8252100]]
SRGB50 = [[0.4360747, 0.3850649, 0.1430804], [0.2225045, 0.7168786, 0.0606169], [0.0139322, 0.0971045, 0.7141733]]


def _mul(a, b):
    """DNGMatrix * DNGMatrix: each entry summed from 0.0 in index order."""
    r = [[0.0] * 3 for _ in range(3)]
    for j in range(3):
        for k in range(3):
            s = 0.0
            for m in range(3):
                s += a[j][m] * b[m][k]
            r[j][k] = s
    return r


def _inv3(m):
    """DNGMatrix.Invert3x3: adjugate / determinant."""
    (a00, a01, a02), (a10, a11, a12), (a20, a21, a22) = m
    t = [[a11 * a22 - a21 * a12, a21 * a02 - a01 * a22, a01 * a12 - a11 * a02],
         [a20 * a12 - a10 * a22, a00 * a22 - a20 * a02, a10 * a02 - a00 * a12],
         [a10 * a21 - a20 * a11, a20 * a01 - a00 * a21, a00 * a11 - a10 * a01]]
    det = a00 * t[0][0] + a01 * t[1][0] + a02 * t[2][0]
    if abs(det) < 1e-10:
        raise ValueError("singular")
    return [[t[j][k] / det for k in range(3)] for j in range(3)]


def _color_space(to_pcs):
    """DNGColorSpace(toPCS): rows scaled to map RGB white to the D50 PCS white."""
    x, y = 0.3457, 0.3585
    w2 = [x / y, 1.0, (1.0 - x - y) / y]
    to = []
    for j in range(3):
        w1 = 0.0
        for m in range(3):
            w1 += to_pcs[j][m] * 1.0
        s = w2[j] / w1
        to.append([s * to_pcs[j][k] for k in range(3)])
    return to, _inv3(to)


def _twist(m):
    t = np.zeros((3, 4), f32)
    for i in range(3):
        for j in range(3):
            t[i, j] = f32(m[i][j])
    return t


def color_twists(camera_to_pcs):
    """(twist camera -> ProPhoto, twist ProPhoto -> sRGB50), float32 3 x 4 each."""
    cam = [[float(camera_to_pcs[j][k]) for k in range(3)] for j in range(3)]
    pp_to, pp_from = _color_space(PROPHOTO)
    s_to, s_from = _color_space(SRGB50)
    return _twist(_mul(pp_from, cam)), _twist(_mul(s_from, pp_to))


def _thr(v, hi):
    v = v.copy()
    v[v < 0] = f32(0)
    hi = np.broadcast_to(np.asarray(hi, f32), v.shape)
    m = v > hi
    v[m] = hi[m]
    return v


def _twist_apply(t, r, g, b):
    out = []
    for i in range(3):
        out.append(((t[i, 0] * r + t[i, 1] * g) + t[i, 2] * b) + t[i, 3])
    return out


def lut_segment(lx, v):
    """Largest k in [0, n - 2] with lx[k] <= v; 0 below the first level and for NaN."""
    n = len(lx)
    k = np.searchsorted(lx, v, side="right").astype(np.int64) - 1
    k[np.isnan(v)] = 0
    return np.clip(k, 0, n - 2)


def lut_coefficients(lx, ly):
    """Per segment k: the cubic through levels i0 .. i0 + 3, i0 = clamp(k - 1, 0, n - 4),
    as float32 (c0, c1, c2, c3) in t = v - lx[k]: Newton divided differences in
    float64 on z_j = lx[i0 + j] - lx[k], expanded from the inside out."""
    lx = np.asarray(lx, f32)
    ly = np.asarray(ly, f32)
    n = len(lx)
    c = np.zeros((n - 1, 4), f32)
    for k in range(n - 1):
        i0 = min(max(k - 1, 0), n - 4)
        z = [float(lx[i0 + j]) - float(lx[k]) for j in range(4)]
        a = [float(ly[i0 + j]) for j in range(4)]
        for o in range(1, 4):
            for j in range(3, o - 1, -1):
                a[j] = (a[j] - a[j - 1]) / (z[j] - z[j - o])
        p = [a[3], 0.0, 0.0, 0.0]
        deg = 0
        for j in (2, 1, 0):
            q = [0.0, 0.0, 0.0, 0.0]
            for d in range(deg + 1):
                q[d + 1] += p[d]
                q[d] -= z[j] * p[d]
            q[0] += a[j]
            deg += 1
            p = q
        c[k] = np.array(p, np.float64).astype(f32)
    return c


def lut_cubic(lx, ly, v, coef=None):
    """The cubic through the four nearest levels, Horner's rule in t = v - lx[k]."""
    lx = np.asarray(lx, f32)
    c = lut_coefficients(lx, ly) if coef is None else coef
    k = lut_segment(lx, v)
    t = v - lx[k]
    ck = c[k]
    return ((ck[..., 3] * t + ck[..., 2]) * t + ck[..., 1]) * t + ck[..., 0]


_GAMMA = None


def gamma_srgb(v):
    """GammasRGB per channel: NaN -> 0, clamp to [0, 1], sRGB curve (kernel.cu:290-332),
    through orc_gamma_srgb_f32 of the oracle library (the C library's powf, as the
    reference's float code; numpy's vectorised float32 power rounds differently)."""
    global _GAMMA
    if _GAMMA is None:
        import ctypes
        import os
        lib = ctypes.CDLL(os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "liboracle64.so"))
        _GAMMA = lib.orc_gamma_srgb_f32
        _GAMMA.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        _GAMMA.restype = None
    a = np.ascontiguousarray(v, f32).copy()
    _GAMMA(a.ctypes.data, a.size)
    return a


def postprocess(img, crop, camera_white, twist1, twist2, lut_x, lut_y, exposure, fmt=0):
    """img: float32 H x W x 3. fmt 0: uint16 RGB crop; 1: uint8 BGRA crop."""
    x0, y0, w, h = crop
    v = np.asarray(img, f32)[y0:y0 + h, x0:x0 + w]
    r, g, b = (_thr(v[..., c], f32(camera_white[c])) for c in range(3))
    r, g, b = _twist_apply(np.asarray(twist1, f32).reshape(3, 4), r, g, b)
    coef = lut_coefficients(lut_x, lut_y)
    r, g, b = (lut_cubic(lut_x, lut_y, _thr(c, f32(1)), coef) for c in (r, g, b))
    amp = f32(2.0 ** float(exposure))
    r, g, b = (c * amp for c in _twist_apply(np.asarray(twist2, f32).reshape(3, 4), r, g, b))
    full, cap = (f32(65535), 65535) if fmt == 0 else (f32(255), 255)

    def conv(c):
        q = gamma_srgb(c) * full
        q = np.where(np.isnan(q), f32(0), q)
        return np.clip(np.rint(q), 0, cap).astype(np.uint16 if fmt == 0 else np.uint8)

    R, G, B = conv(r), conv(g), conv(b)
    if fmt == 0:
        return np.stack([R, G, B], -1)
    return np.stack([B, G, R, np.full_like(R, 255)], -1)


def tiff16_bytes(rgb):
    """The bytes SaveAsTiff writes for a uint16 H x W x 3 image."""
    rgb = np.asarray(rgb, np.uint16)
    h, w, _ = rgb.shape
    entries = [  # tag, type, count, inline value or out-of-line payload
        (256, 4, 1, w), (257, 4, 1, h), (258, 3, 3, struct.pack("<3H", 16, 16, 16)), (259, 3, 1, 1), (262, 3, 1, 2),
        (273, 4, 1, None), (277, 3, 1, 3), (278, 4, 1, h), (279, 4, 1, w * h * 6), (282, 5, 1, struct.pack("<2I", 720, 10)),
        (283, 5, 1, struct.pack("<2I", 720, 10)), (296, 3, 1, 1), (271, 2, 8, b"MK TIFF\0")]
    ifd_end = 8 + 2 + 12 * len(entries) + 4
    tail = b""
    recs = []
    for tag, typ, cnt, val in entries:
        if isinstance(val, bytes):
            recs.append([tag, typ, cnt, ifd_end + len(tail)])
            tail += val
        else:
            recs.append([tag, typ, cnt, val])
    data_at = ifd_end + len(tail)
    for r in recs:
        if r[0] == 273:
            r[3] = data_at
    out = b"II*\0" + struct.pack("<I", 8) + struct.pack("<H", len(recs))
    out += b"".join(struct.pack("<HHII", *r) for r in recs) + b"\0\0\0\0" + tail
    return out + rgb.astype("<u2").tobytes()


def parse_tiff16(buf):
    """Minimal reader for the layout above: (tags {tag: (type, count, value/offset)}, image)."""
    assert buf[:4] == b"II*\0"
    (off,) = struct.unpack_from("<I", buf, 4)
    (n,) = struct.unpack_from("<H", buf, off)
    tags = {}
    for i in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", buf, off + 2 + 12 * i)
        tags[tag] = (typ, cnt, val)
    w, h = tags[256][2], tags[257][2]
    at, nb = tags[273][2], tags[279][2]
    img = np.frombuffer(buf, "<u2", count=nb // 2, offset=at).reshape(h, w, 3)
    return tags, img
