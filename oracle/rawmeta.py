"""CPU restatement of the raw-file metadata (test infrastructure: only tests/
use it): the levels and geometry of DNGFile.SetMembers
(PefFile/DNGFile.cs:706-967) and of the DNGFile constructor (:288-372,
:607-609), NoiseModel.GetValue (PefFile/ExtraCameraProfiles.cs:164-199) and
the crop rule of RawFile.LoadExtraCameraProfile (PefFile/RawFile.cs:246-261),
in the reference's order with C#'s float / double conversions.

Parity is unpinned: the C# cannot run here and the reference's tests hold no
metadata vectors; libisa.so's host code is checked against this restatement
field by field.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


class ReferenceThrows(Exception):
    """Where the reference raises (ArgumentException, IndexOutOfRange, ...)."""


def noise_model(iso, isos, alpha, beta):
    """NoiseModel.GetValue: the last profile ISO not above `iso`, linear to the next one."""
    if len(isos) == 0:
        return 0.0, 0.0
    index = -1
    for i in range(len(isos) - 1, -1, -1):
        if isos[i] <= iso:
            index = i
            break
    if index == len(isos) - 1:
        return float(alpha[-1]), float(beta[-1])
    if index < 0:
        return float(alpha[0]), float(beta[0])
    w = (float(iso) - float(isos[index + 1])) / (float(isos[index]) - float(isos[index + 1]))
    return w * float(alpha[index]) + (1.0 - w) * float(alpha[index + 1]), w * float(beta[index]) + (1.0 - w) * float(beta[index + 1])


def crop_window(left, top, cw, ch, width, height):
    """At least two pixels off the left / top; the size ends two pixels before the right / bottom."""
    return (max(2, left), max(2, top), cw - max(0, (left + cw) - (width - 2)), ch - max(0, (top + ch) - (height - 2)))


def _trunc(v):
    return int(math.trunc(float(v)))


def _cs_max(a, b):
    if np.isnan(a) or np.isnan(b):
        return f32(np.nan)
    return a if a > b else b


def dng_levels(width, height, cfa_pattern, white_level, camera_white, cfa_repeat=(2, 2), plane_color=None, black_level=None,
               active_area=None, default_crop_origin=None, default_crop_size=None, noise_profile=None, black_delta_h=None,
               black_delta_v=None, iso=0, profile_noise=None):
    """The values DNGFile leaves in RawFile's fields, as a dict (see isa.dng_levels)."""
    if tuple(cfa_repeat) != (2, 2):
        raise ReferenceThrows("bayer pattern size different than 2x2")
    bayer = [int(c) for c in cfa_pattern]
    if any(c not in (0, 1, 2) for c in bayer):
        raise ReferenceThrows("CFA colour other than red, green, blue")
    helper = [0, 1, 2]
    twist = np.zeros((3, 4), f32)
    twist[0, 0] = twist[1, 1] = twist[2, 2] = 1
    identity = True
    if plane_color is not None:
        twist = np.zeros((3, 4), f32)
        if len(plane_color) != 3:
            raise ReferenceThrows("not three colour planes")
        for i, color in enumerate(plane_color):
            helper[i] = int(color)
            if not 0 <= color <= 2:
                raise ReferenceThrows("colour other than red/green/blue")
            twist[color, i] = 1
            if color != i:
                identity = False
    black = [f32(0)] * 3
    if black_level is not None:
        bl = [f32(v) for v in black_level]
        if len(bl) == 1:
            black = [bl[0]] * 3
        elif len(bl) == 3:
            black = list(black)
            for i in range(3):
                black[helper[i]] = bl[i]
        elif len(bl) == 4:
            try:
                ir = bayer.index(0)
                ib = bayer.index(2)
            except ValueError:
                raise ReferenceThrows("index -1")
            g1 = g2 = -1
            for i in range(4):
                if bayer[i] == 1 and g1 == -1:
                    g1 = i
                if bayer[i] == 1 and g1 != -1:
                    g2 = i
            if g1 < 0:
                raise ReferenceThrows("index -1")
            black = [bl[ir], _cs_max(bl[g1], bl[g2]), bl[ib]]
    wl = f32(white_level)
    white = [f32(wl - black[c]) for c in range(3)]
    wb = [f32(0)] * 3
    for i in range(3):
        wb[helper[i]] = f32(f32(1.0) / f32(camera_white[i]))
    crop_left = crop_top = 0
    cw, ch = width, height
    if active_area is not None:
        top, left, bottom, right = (int(v) for v in active_area)
        crop_left += left
        crop_top += top
        cw, ch = right - left, bottom - top
        if math.fmod(top, 2) != 0:
            bayer = [bayer[2], bayer[3], bayer[0], bayer[1]]
        if math.fmod(left, 2) != 0:
            bayer = [bayer[1], bayer[0], bayer[3], bayer[2]]
    if default_crop_origin is not None and default_crop_size is not None:
        left = top = _trunc(default_crop_origin[0])
        w = h = _trunc(default_crop_size[0])
        crop_left += left
        crop_top += top
        cw, ch = w, h
    crop = crop_window(crop_left, crop_top, cw, ch, width, height)
    alpha = beta = f32(0)
    if noise_profile is not None:
        if len(noise_profile) < 2 or (len(noise_profile) > 2 and len(noise_profile) < helper[1] * 2 + 2):
            raise ReferenceThrows("index outside NoiseProfile")
        if len(noise_profile) > 2:
            alpha, beta = f32(noise_profile[helper[1] * 2]), f32(noise_profile[helper[1] * 2 + 1])
        else:
            alpha, beta = f32(noise_profile[0]), f32(noise_profile[1])
    if profile_noise is not None:
        a, b = noise_model(iso, *profile_noise)
        if a != 0.0:
            alpha, beta = f32(a), f32(b)
    off_v = off_h = 0
    border_bottom = border_right = 0
    if active_area is not None:
        off_v, off_h = int(active_area[0]), int(active_area[1])
        border_bottom, border_right = height - int(active_area[2]), width - int(active_area[3])
    bv = np.zeros(height, np.uint16)
    bh = np.zeros(width, np.uint16)
    if black_delta_v is not None:
        if len(black_delta_v) + off_v + border_bottom != height:
            raise ReferenceThrows("BlackLevelDeltaV doesn't fit")
        for i, v in enumerate(black_delta_v):
            bv[off_v + i] = _trunc(v)
    if black_delta_h is not None:
        if len(black_delta_h) + off_h + border_right != width:
            raise ReferenceThrows("BlackLevelDeltaH doesn't fit")
        for i, v in enumerate(black_delta_h):
            bh[off_h + i] = _trunc(v)
    # the largest black of any decoded pixel (every pixel of the frame is decoded)
    max_black = max(int(bh[c]) + int(bv[r]) for r in range(height) for c in range(width)) if width * height <= 65536 else \
        int(bh.max()) + int(bv.max())
    white = [f32(w - f32(max_black)) for w in white]
    return dict(cfa=bayer, black=np.array(black, f32), white=np.array(white, f32), camera_white=np.array([f32(v) for v in camera_white], f32),
                noise=(f32(alpha), f32(beta)), white_balance=np.array(wb, f32), color_twist=twist, color_twist_identity=identity,
                crop=tuple(crop), black_h=bh, black_v=bv)
