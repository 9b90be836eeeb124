"""CPU merge pipeline over the checkers -- TEST INFRASTRUCTURE ONLY.

Drives a whole burst merge the way the reference controller does
(PEFStudioDX/ImageStackAlignatorController.cs: DeBayerBWGaussWB :2384-2418,
TrackPatches :1601-1746, PrepareAccumulation :1795-1926, Accumulate
:1928-1987) on one of three stage libraries:

  "oracle64" -- the FP64 restatement (oracle/isa_oracle.c),
  "ref64"    -- the reference's own kernel bodies with float -> double,
  "ref32"    -- the reference's own kernel bodies in float (the timed host
                baseline; OpenMP over grid blocks).

Library steps with no reference source (NPP filters, resize, erode, the
cuBLAS solve) come from isa_oracle.c in the matching precision; the
full-frame FFT of the high-pass is numpy's. Only tests, the smoke check and
bench.py's CPU baseline import this module.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from imagestackalignator_b200 import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def _load(path):
    if path not in _LIBS:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        _LIBS[path] = ctypes.CDLL(path)
    return _LIBS[path]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class StageLib:
    """numpy front end over one checker library."""

    def __init__(self, kind="oracle64"):
        self.kind = kind
        if kind == "oracle64":
            self.k = _load(os.path.join(HERE, "_build", "liboracle64.so"))
            self.lib = self.k
            self.dtype = np.float64
            self.pfx = "orc_"
        elif kind in ("ref32", "ref64"):
            self.k = _load(os.path.join(HERE, "_ref", f"lib{kind}.so"))
            self.lib = _load(os.path.join(HERE, "_build", "liboracle32.so" if kind == "ref32" else "liboracle64.so"))
            self.dtype = np.float32 if kind == "ref32" else np.float64
            self.pfx = "ref_"
        else:
            raise ValueError(kind)
        self.R = ctypes.c_float if self.dtype == np.float32 else ctypes.c_double

    # helpers --------------------------------------------------------------
    def arr(self, a):
        return np.ascontiguousarray(a, dtype=self.dtype)

    def vec(self, v):
        return np.ascontiguousarray(np.asarray(v, dtype=self.dtype))

    def kf(self, name):
        return getattr(self.k, self.pfx + name)

    def lf(self, name):
        return getattr(self.lib, "orc_" + name)

    def set_threads(self, n):
        if self.kind.startswith("ref"):
            self.k.ref_set_threads(ctypes.c_int(n))

    # kernels (reference bodies or restatement) -----------------------------
    def debayer_full(self, raw, cfa, black, scale, divisor):
        H, W = raw.shape
        out = np.empty((H, W, 3), self.dtype)
        c = np.ascontiguousarray(cfa, dtype=np.int32)
        self.kf("debayer_full")(_p(np.ascontiguousarray(raw)), W, H, _p(c), _p(self.vec(black)), _p(self.vec(scale)),
                                _p(self.vec(divisor)), _p(out))
        return out

    def gamma_srgb(self, rgb):
        rgb = self.arr(rgb).copy()
        H, W, _ = rgb.shape
        self.kf("gamma_srgb")(_p(rgb), W, H)
        return rgb

    def fourier_mask(self, W, H, lp, hp, lps, hps, clear_axis):
        m = np.empty((H, W // 2 + 1), self.dtype)
        R = self.R
        self.kf("fourier_filter_mask")(W, H, R(lp), R(hp), R(lps), R(hps), clear_axis, _p(m))
        return m

    def track_pair(self, img_trk, img_ref, T, S, tcx, tcy, pre, base_ref, rot_ref, base_trk, rot_trk, thr, want_scores=False,
                   want_offsets=False):
        """Returns (pre + shift, L2 maps or None), plus the unrounded search
        block offsets (tiles x 2) when want_offsets (restatement only)."""
        Hl, Wl = img_trk.shape
        pre = self.arr(pre).copy()
        D = 2 * S + 1
        scores = np.empty((tcy * tcx, D * D), self.dtype) if want_scores else None
        offs = np.empty((tcy * tcx, 2), self.dtype) if want_offsets else None
        R = self.R
        args = [_p(self.arr(img_trk)), _p(self.arr(img_ref)), Wl, Hl, T, S, tcx, tcy, _p(pre), _p(self.vec(base_ref)), R(rot_ref),
                _p(self.vec(base_trk)), R(rot_trk), R(thr), _p(scores)]
        if self.pfx == "orc_":
            args += [None, _p(offs)]
        elif want_offsets:
            raise ValueError("offsets come from the restatement only")
        self.kf("track_pair")(*args)
        if want_offsets:
            return pre, scores, offs
        return pre, scores

    def upsample_shifts(self, grid, old_level, new_level, ncx, ncy, old_t, new_t):
        ocy, ocx, _ = grid.shape
        out = np.empty((ncy, ncx, 2), self.dtype)
        self.kf("upsample_shifts")(_p(self.arr(grid)), _p(out), old_level, new_level, ocx, ocy, ncx, ncy, old_t, new_t)
        return out

    def solve_shifts(self, A, meas):
        tiles, m, _ = meas.shape
        n1 = A.shape[1]
        meas = self.arr(meas).copy()
        x = np.empty((tiles, n1, 2), self.dtype)
        st = np.empty(tiles, np.int32)
        fn = self.k.ref_solve_shifts if self.pfx == "ref_" else self.k.orc_solve_shifts
        fn(_p(self.arr(A)), m, n1, tiles, _p(meas), _p(x), _p(st))
        return meas, x, st

    def optimal_shifts(self, x, tcx, tcy, ref, trk):
        tiles, n1, _ = x.shape
        out = np.empty((tcy, tcx, 2), self.dtype)
        if self.pfx == "ref_":
            self.k.ref_optimal_shifts(_p(self.arr(x)), n1, tcx, tcy, ref, trk, _p(out))
        else:
            self.k.orc_optimal_shifts(_p(self.arr(x)), n1, tiles, ref, trk, _p(out))
        return out

    def flow_from_tiles(self, tiles, W, H, base, rot, T):
        tcy, tcx, _ = tiles.shape
        out = np.empty((H, W, 2), self.dtype)
        if self.pfx == "ref_":
            self.k.ref_flow_from_tiles(_p(self.arr(tiles)), tcx, tcy, W, H, _p(self.vec(base)), self.R(rot), T, _p(out))
        else:
            self.k.orc_flow_from_tiles(_p(self.arr(tiles)), tcx, tcy, W, H, _p(self.vec(base)), self.R(rot), _p(out))
        return out

    def warp(self, img, flow):
        H, W = img.shape
        out = np.empty((H, W), self.dtype)
        self.kf("warp")(_p(self.arr(img)), W, H, _p(self.arr(flow)), _p(out))
        return out

    def derivatives(self, src, tgt):
        H, W = src.shape
        ix, iy, it = (np.empty((H, W), self.dtype) for _ in range(3))
        self.kf("derivatives")(_p(self.arr(src)), _p(self.arr(tgt)), W, H, _p(ix), _p(iy), _p(it))
        return ix, iy, it

    def derivatives2(self, img):
        H, W = img.shape
        ix, iy = (np.empty((H, W), self.dtype) for _ in range(2))
        self.kf("derivatives2")(_p(self.arr(img)), W, H, _p(ix), _p(iy))
        return ix, iy

    def lucas_kanade(self, flow, ix, iy, it, half, min_det):
        H, W = ix.shape
        flow = self.arr(flow).copy()
        self.kf("lucas_kanade")(_p(flow), _p(self.arr(ix)), _p(self.arr(iy)), _p(self.arr(it)), W, H, half, self.R(min_det))
        return flow

    def debayer_subsample(self, raw, cfa, max_val):
        H, W = raw.shape
        out = np.empty((H // 2, W // 2, 3), self.dtype)
        c = np.ascontiguousarray(cfa, dtype=np.int32)
        self.kf("debayer_subsample")(_p(np.ascontiguousarray(raw)), W, H, _p(c), self.R(max_val), _p(out))
        return out

    def robustness_mask(self, ref, mov, flow, alpha, beta, thr_m, mask, s=1.5, t=float(np.float32(0.12)), bilinear=False):
        Hh, Wh, _ = ref.shape
        Hf, Wf, _ = flow.shape
        mask = self.arr(mask).copy()
        R = self.R
        if self.pfx == "ref_":
            self.k.ref_robustness_mask(_p(self.arr(ref)), _p(self.arr(mov)), Wh, Hh, _p(self.arr(flow)), Wf, Hf, R(alpha), R(beta),
                                       R(thr_m), _p(mask))
        else:
            fn = self.k.orc_robustness_mask_bil if bilinear else self.k.orc_robustness_mask
            fn(_p(self.arr(ref)), _p(self.arr(mov)), Wh, Hh, _p(self.arr(flow)), Wf, Hf, R(alpha), R(beta), R(thr_m), R(s), R(t), _p(mask))
        return mask

    def structure_tensor(self, dx, dy):
        H, W = dx.shape
        out = np.empty((H, W, 3), self.dtype)
        self.kf("structure_tensor")(_p(self.arr(dx)), _p(self.arr(dy)), W, H, _p(out))
        return out

    def kernel_param(self, st, p: P.MergeParams):
        st = self.arr(st).copy()
        H, W, _ = st.shape
        R = self.R
        self.kf("kernel_param")(_p(st), W, H, R(p.f32("dth")), R(p.f32("dtr")), R(p.f32("k_detail")), R(p.f32("k_denoise")),
                                R(p.f32("k_stretch")), R(p.f32("k_shrink")))
        return st

    def apply_weighting(self, img, acc, wsum, thr):
        img = self.arr(img).copy()
        H, W, _ = img.shape
        self.kf("apply_weighting")(_p(img), _p(self.arr(acc)), _p(self.arr(wsum)), W, H, self.R(thr))
        return img

    def accumulate(self, raw, cfa, acc, wsum, mask, kparam, flow, white, black, scale, origin, crop, bilinear=False):
        """Generalised scale-s accumulation (restatement only); bilinear: sample mode BILINEAR."""
        H, W = raw.shape
        Ho, Wo, _ = acc.shape
        c = np.ascontiguousarray(cfa, dtype=np.int32)
        cr = np.ascontiguousarray(crop, dtype=np.int32)
        kparam = self.arr(kparam)
        fn = self.k.orc_accumulate_bil if bilinear else self.k.orc_accumulate
        fn(_p(np.ascontiguousarray(raw)), W, H, _p(c), _p(acc), _p(wsum), Wo, Ho, _p(self.arr(mask)), _p(kparam), kparam.shape[2],
           _p(self.arr(flow)), _p(self.vec(white)), _p(self.vec(black)), self.R(scale), origin[0], origin[1], _p(cr))

    def accumulate_ref(self, raw, cfa, acc, wsum, mask, kparam, flow, white, black, superres):
        H, W = raw.shape
        c = np.ascontiguousarray(cfa, dtype=np.int32)
        fn = self.k.ref_accumulate_superres if superres else self.k.ref_accumulate
        fn(_p(np.ascontiguousarray(raw)), W, H, _p(c), _p(acc), _p(wsum), _p(self.arr(mask)), _p(self.arr(kparam)),
           _p(self.arr(flow)), _p(self.vec(white)), _p(self.vec(black)))

    # library steps (restated NPP / host code) -------------------------------
    def color_to_gray(self, rgb, w):
        H, W, _ = rgb.shape
        out = np.empty((H, W), self.dtype)
        self.lf("color_to_gray")(_p(self.arr(rgb)), W, H, _p(self.vec(w)), _p(out))
        return out

    def clamp01(self, img):
        img = self.arr(img).copy()
        self.lf("clamp01")(_p(img), ctypes.c_size_t(img.size))
        return img

    def gauss_taps(self, sigma):
        """gaussian_filter_1D (controller :2351-2382), computed in float like the C# host."""
        sigma = np.float32(sigma)
        if sigma <= 0:
            t = np.zeros(9, np.float32); t[4] = 1
            return t.astype(self.dtype)
        size = int(np.float32(sigma / np.float32(0.6)) - np.float32(0.4)) * 2 + 1 + 2
        size = min(size, 99)
        c = size // 2
        if self.dtype == np.float32:
            t = np.array([np.float32(np.exp(np.float64(np.float32(-((i - c) * (i - c))) / (np.float32(2) * sigma * sigma))))
                          for i in range(size)], np.float32)
            s = np.float32(0)
            for v in t:
                s = np.float32(s + v)
            return (t / s).astype(np.float32)
        t = np.empty(99, np.float64)
        n = self.lib.orc_gauss_taps(ctypes.c_double(float(sigma)), _p(t))
        return t[:n].copy()

    def gauss_filter(self, img, taps):
        img = self.arr(img)
        H, W = img.shape[:2]
        C = 1 if img.ndim == 2 else img.shape[2]
        out = np.empty_like(img)
        taps = self.vec(taps)
        self.lf("gauss_filter")(_p(img), W, H, C, _p(taps), len(taps), _p(out))
        return out

    def resize_box(self, img, L):
        H, W = img.shape
        out = np.empty((H // L, W // L), self.dtype)
        self.lf("resize_box")(_p(self.arr(img)), W, H, L, _p(out))
        return out

    def erode(self, img, size):
        img = self.arr(img)
        H, W, C = img.shape
        out = np.empty_like(img)
        self.lf("erode")(_p(img), W, H, C, size, _p(out))
        return out


# ---------------------------------------------------------------------------
# pipeline
# ---------------------------------------------------------------------------
GRAY_WEIGHTS = (0.2989, 0.5870, 0.1141)


@dataclass
class PreAlignment:
    """PreAlignmentStore state (PreAlignmentStore.cs:27-150): per-frame shift
    and rotation (degrees) and the reference index."""
    shifts: np.ndarray
    rotations: np.ndarray
    reference: int = 0

    @staticmethod
    def zeros(n):
        return PreAlignment(np.zeros((n, 2)), np.zeros(n), 0)

    def shift(self, frm, to):
        return (self.shifts[to] - self.shifts[frm]).astype(np.float32)

    def rotation(self, frm, to):
        return float(np.float32(np.float32(self.rotations[to] - self.rotations[frm]) / np.float32(180.0) * np.float32(np.pi)))


@dataclass
class MergeResult:
    image: np.ndarray
    acc: np.ndarray
    wsum: np.ndarray
    stages: dict = field(default_factory=dict)


def bw_image(lib: StageLib, burst, i, sigma, high_pass: bool, p: P.MergeParams):
    """DeBayerBWGaussWB (controller :2384-2418)."""
    cw = np.asarray(burst.camera_white, np.float64)
    black = np.asarray(burst.black, np.float64)
    white = np.asarray(burst.white, np.float64)
    scale = (1.0 / cw).astype(np.float32)
    divisor = (white.astype(np.float32) / cw.astype(np.float32)).astype(np.float32)
    rgb = lib.debayer_full(burst.raw[i], burst.cfa, black, scale, divisor)
    rgb = lib.gamma_srgb(rgb)
    w = (0.0, 1.0, 0.0) if p.green_channel_only else GRAY_WEIGHTS
    gray = lib.color_to_gray(rgb, np.float32(w))
    H, W = gray.shape
    if high_pass:
        # PreAlignment.FourierFilter (PreAlignment.cs:268-281): R2C, filter
        # (lp = 1, lps = 1), C2R, / (W*H), clamp to [0, 1]
        mask = lib.fourier_mask(W, H, 1.0, p.f32("high_pass"), 1.0, p.f32("high_pass_sigma"), p.clear_axis)
        spec = np.fft.rfft2(gray.astype(np.float64))
        gray = np.fft.irfft2(spec * mask, s=(H, W)).astype(lib.dtype)
        gray = lib.clamp01(gray)
    return lib.gauss_filter(gray, lib.gauss_taps(sigma))


def track_patches(lib: StageLib, bw_track, pre: PreAlignment, p: P.MergeParams, keep=None):
    """TrackPatches (controller :1601-1746)."""
    n, H, W = bw_track.shape
    strat, blk = p.tracking_strategy, p.tracking_block_size
    pairs = P.shift_pairs(n, pre.reference, strat, blk)
    idx = P.index_table(n, pre.reference, strat, blk)
    A = P.shift_matrix(n, pre.reference, strat, blk)
    L = p.levels
    lv0 = L[0]
    maxcx = max((W // l.resize_level - 2 * l.max_shift) // l.tile_size for l in L)
    maxcy = max((H // l.resize_level - 2 * l.max_shift) // l.tile_size for l in L)
    grids = np.zeros((len(pairs), maxcy, maxcx, 2), lib.dtype)
    x = None
    old = None
    for li in range(len(L) - 1, -1, -1):
        lvl = L[li]
        Wl, Hl = W // lvl.resize_level, H // lvl.resize_level
        T, S = lvl.tile_size, lvl.max_shift
        tcx, tcy = (Wl - 2 * S) // T, (Hl - 2 * S) // T
        if old is not None:
            ocx, ocy, olevel, oT = old
            for (r, t) in pairs:
                k = idx[r, t]
                grids[k, :tcy, :tcx] = lib.upsample_shifts(grids[k, :ocy, :ocx], olevel, lvl.resize_level, tcx, tcy, oT, T)
        if lvl.resize_level > 1:
            imgs = np.stack([lib.resize_box(bw_track[f], lvl.resize_level) for f in range(n)])
        else:
            imgs = bw_track
        for (r, t) in pairs:
            k = idx[r, t]
            want_offs = keep is not None and lib.pfx == "orc_"
            res = lib.track_pair(imgs[t], imgs[r], T, S, tcx, tcy, grids[k, :tcy, :tcx],
                                 pre.shift(pre.reference, r) / np.float32(lvl.resize_level), pre.rotation(pre.reference, r),
                                 pre.shift(pre.reference, t) / np.float32(lvl.resize_level), pre.rotation(pre.reference, t),
                                 p.f32("matching_threshold"), want_scores=keep is not None, want_offsets=want_offs)
            g, sc = res[0], res[1]
            grids[k, :tcy, :tcx] = g
            if keep is not None:
                keep.setdefault("scores", {})[(li, r, t)] = sc
                keep.setdefault("measured", {})[(li, r, t)] = g.copy()
                if want_offs:
                    keep.setdefault("offsets", {})[(li, r, t)] = res[2]
        # MinimizeCUBLAS (ShiftCollection.cs:738-822)
        meas = np.stack([grids[idx[r, t], :tcy, :tcx].reshape(-1, 2) for (r, t) in
                         sorted(pairs, key=lambda rt: idx[rt[0], rt[1]])], axis=1)
        meas, x, st = lib.solve_shifts(A, meas)
        for j, (r, t) in enumerate(sorted(pairs, key=lambda rt: idx[rt[0], rt[1]])):
            grids[idx[r, t], :tcy, :tcx] = meas[:, j, :].reshape(tcy, tcx, 2)
        if keep is not None:
            keep.setdefault("solved_x", {})[li] = x.copy()
            keep.setdefault("status", {})[li] = st.copy()
        old = (tcx, tcy, lvl.resize_level, T)
    tcx0 = (W // lv0.resize_level - 2 * lv0.max_shift) // lv0.tile_size
    tcy0 = (H // lv0.resize_level - 2 * lv0.max_shift) // lv0.tile_size
    return x, (tcx0, tcy0)


def out_geometry(W, H, p: P.MergeParams):
    """Output size, scale, origin and crop of the accumulation.
    Reference plain: s = 1 over the frame; reference super-resolution: s = 2
    over the central W/2 x H/2 crop with origin (W/2, H/2)
    (DeBayerKernels.cu:398-423); merge_scale > 0: the whole frame at scale s."""
    if p.merge_scale and p.merge_scale > 0:
        s = float(np.float32(p.merge_scale))
        return int(round(W * s)), int(round(H * s)), s, (0, 0), (0, 0, W - 1, H - 1), 0.0
    if p.super_resolution:
        return W, H, 2.0, (W // 2, H // 2), (W // 4, H // 4, W // 2 - 1 + W // 4, H // 2 - 1 + H // 4), 0.0
    return W, H, 1.0, (0, 0), (0, 0, W - 1, H - 1), 1.0


def merge_burst(burst, p: P.MergeParams = None, kind="oracle64", pre: Optional[PreAlignment] = None,
                keep: Optional[dict] = None, threads=0, lib: Optional[StageLib] = None, tiles: Optional[dict] = None):
    """Whole forward merge of one burst. Returns MergeResult (FP arrays of the
    backend's precision). `keep`, when a dict, receives intermediates.
    `tiles` (frame -> tiles_y x tiles_x x 2) replaces the solved tile flows,
    as isa_set_tile_flow does; p.sample_mode SAMPLE_BILINEAR selects the
    blended accumulation and mask (restatement only)."""
    p = p or P.MergeParams()
    lib = lib or StageLib(kind)
    bil = p.sample_mode == P.SAMPLE_BILINEAR
    if bil and lib.pfx != "orc_":
        raise ValueError("sample mode BILINEAR has no counterpart in the reference's kernels")
    if threads:
        lib.set_threads(threads)
    n, H, W = burst.raw.shape
    pre = pre or PreAlignment.zeros(n)
    ref = pre.reference
    # tracking images (SkipPreAlignment / ComputePreAlignment :1554-1557)
    bw_track = np.stack([bw_image(lib, burst, i, p.sigma_debayer_tracking, True, p) for i in range(n)])
    x, (tcx0, tcy0) = track_patches(lib, bw_track, pre, p, keep)
    # PrepareAccumulation (:1795-1926)
    bw_acc = np.stack([bw_image(lib, burst, i, p.sigma_debayer_accumulation, False, p) for i in range(n)])
    dx, dy = lib.derivatives2(bw_acc[ref])
    st = lib.structure_tensor(dx, dy)
    st = lib.gauss_filter(st, lib.gauss_taps(p.sigma_structure_tensor))
    kparam = lib.kernel_param(st, p)
    white = np.asarray(burst.white, np.float64)
    black = np.asarray(burst.black, np.float64)
    max_val = float(np.max(np.float32(white) + np.float32(black)))
    ref_half = lib.debayer_subsample(burst.raw[ref], burst.cfa, max_val)
    Wo, Ho, s, origin, crop, thr = out_geometry(W, H, p)
    acc = np.zeros((Ho, Wo, 3), lib.dtype)
    wsum = np.zeros((Ho, Wo, 3), lib.dtype)
    ones = np.ones((H // 2, W // 2, 4), lib.dtype)
    zero_flow = np.zeros((H, W, 2), lib.dtype)
    use_canvas = lib.pfx == "ref_" and p.merge_scale and p.merge_scale > 0
    kp4 = np.concatenate([kparam, np.zeros((H, W, 1), lib.dtype)], axis=2)

    def accumulate(raw_i, mask_i, flow_i):
        if lib.pfx == "orc_":
            lib.accumulate(raw_i, burst.cfa, acc, wsum, mask_i, kparam, flow_i, white, black, s, origin, crop, bilinear=bil)
        elif not use_canvas:
            lib.accumulate_ref(raw_i, burst.cfa, acc, wsum, mask_i, kp4 if p.super_resolution else kparam, flow_i, white, black,
                               p.super_resolution)
        else:
            accumulate_canvas_ref(lib, raw_i, burst.cfa, acc, wsum, mask_i, kp4, flow_i, white, black, s)

    accumulate(burst.raw[ref], ones, zero_flow)
    # Accumulate (:1928-1987)
    mask = np.ones((H // 2, W // 2, 4), lib.dtype)
    lv0 = p.levels[0]
    for i in range(n):
        if i == ref:
            continue
        mov_half = lib.debayer_subsample(burst.raw[i], burst.cfa, max_val)
        tiles_i = lib.arr(tiles[i]) if tiles is not None else lib.optimal_shifts(x, tcx0, tcy0, ref, i)
        flow = lib.flow_from_tiles(tiles_i, W, H, pre.shift(ref, i), pre.rotation(ref, i), lv0.tile_size)
        for _ in range(p.iterations_lk):
            warped = lib.warp(bw_acc[i], flow)
            ix, iy, it = lib.derivatives(warped, bw_acc[ref])
            flow = lib.lucas_kanade(flow, ix, iy, it, p.window_size_lk // 2, p.f32("min_det_lk"))
        mask = lib.robustness_mask(ref_half, mov_half, flow, float(np.float32(burst.noise_a)), float(np.float32(burst.noise_b)),
                                   p.f32("threshold_m"), mask, p.f32("robust_s"), p.f32("robust_t"), bilinear=bil)
        eroded = lib.erode(mask, p.erode_size)
        if keep is not None:
            keep.setdefault("flow", {})[i] = flow
            keep.setdefault("mask", {})[i] = eroded
            keep.setdefault("tiles", {})[i] = tiles_i
            keep.setdefault("tail_flow", {}).setdefault(i, (np.array(tiles_i, copy=True), flow))
        accumulate(burst.raw[i], eroded, flow)
    if thr > 0:
        cw = np.asarray(burst.camera_white, np.float64)
        dec = lib.debayer_full(burst.raw[ref], burst.cfa, black, (1.0 / cw).astype(np.float32),
                               (white.astype(np.float32) / cw.astype(np.float32)))
    else:
        dec = np.zeros((Ho, Wo, 3), lib.dtype)
    image = lib.apply_weighting(dec, acc, wsum, thr)
    if keep is not None:
        keep["bw_track"] = bw_track
        keep["bw_acc"] = bw_acc
        keep["kparam"] = kparam
        keep["x"] = x
    return MergeResult(image=image, acc=acc, wsum=wsum)


def merge_tail(burst, p: P.MergeParams, flows, masks, kparam, lib: StageLib, reference=0):
    """The accumulation and ApplyWeighting of a burst (PrepareAccumulation
    :1894-1902, Accumulate :1978-1986, ApplyWeighting :1994-2002) on given
    per-frame flows and eroded masks (dicts frame -> array, the reference
    frame excluded) and kernel parameters, in the restatement's precision.
    The parity checker feeds it the GPU's flows and masks to separate the
    accumulation's own arithmetic from upstream FP32 differences."""
    n, H, W = burst.raw.shape
    white = np.asarray(burst.white, np.float64)
    black = np.asarray(burst.black, np.float64)
    Wo, Ho, s, origin, crop, thr = out_geometry(W, H, p)
    acc = np.zeros((Ho, Wo, 3), lib.dtype)
    wsum = np.zeros((Ho, Wo, 3), lib.dtype)
    kparam = lib.arr(kparam)
    bil = p.sample_mode == P.SAMPLE_BILINEAR
    lib.accumulate(burst.raw[reference], burst.cfa, acc, wsum, np.ones((H // 2, W // 2, 4), lib.dtype), kparam,
                   np.zeros((H, W, 2), lib.dtype), white, black, s, origin, crop, bilinear=bil)
    for i in range(n):
        if i == reference:
            continue
        lib.accumulate(burst.raw[i], burst.cfa, acc, wsum, lib.arr(masks[i]), kparam, lib.arr(flows[i]), white, black, s, origin, crop,
                       bilinear=bil)
    if thr > 0:
        cw = np.asarray(burst.camera_white, np.float64)
        dec = lib.debayer_full(burst.raw[reference], burst.cfa, black, (1.0 / cw).astype(np.float32),
                               (white.astype(np.float32) / cw.astype(np.float32)))
    else:
        dec = np.zeros((Ho, Wo, 3), lib.dtype)
    return MergeResult(image=lib.apply_weighting(dec, acc, wsum, thr), acc=acc, wsum=wsum)


def merge_from_tiles(burst, p: P.MergeParams, tiles, keep, lib: StageLib, pre: Optional[PreAlignment] = None):
    """The merge from given per-frame tile flows on (frame -> tiles_y x
    tiles_x x 2): flow from tiles, LK, robustness mask and erosion (Accumulate
    :1961-1977), kernel parameters, accumulation and ApplyWeighting, reusing
    the reference frame's accumulation image of an earlier merge_burst of the
    same burst (keep["bw_acc"]). Equal to merge_burst(..., tiles=tiles)
    without its tile alignment; the finite differences of the tile-flow and
    parameter gradients evaluate it.

    Each frame's flow (which depends on its tile flow), mask (also on
    robust_s, robust_t) and accumulation sums (also on the kernel parameters)
    of the first call are cached in keep, so that a call that changes one
    frame's tile flow, or only the mask or kernel parameters, recomputes only
    what depends on the change. The frames' sums are added in frame order
    (merge_burst's running sums up to FP64 rounding)."""
    n, H, W = burst.raw.shape
    pre = pre or PreAlignment.zeros(n)
    ref = pre.reference
    bw_acc = keep["bw_acc"]
    white = np.asarray(burst.white, np.float64)
    black = np.asarray(burst.black, np.float64)
    max_val = float(np.max(np.float32(white) + np.float32(black)))
    bil = p.sample_mode == P.SAMPLE_BILINEAR
    Wo, Ho, s, origin, crop, thr = out_geometry(W, H, p)
    if thr > 0:
        raise ValueError("merge_from_tiles covers the merge_scale and super-resolution modes (normalisation threshold 0)")
    kkey = tuple(p.f32(k) for k in ("dth", "dtr", "k_detail", "k_denoise", "k_stretch", "k_shrink")) + (p.sigma_structure_tensor,)
    mkey = (p.f32("robust_s"), p.f32("robust_t"))
    kp = keep.setdefault("tail_kparam", {})
    if kkey not in kp:
        if len(kp) >= 2:
            kp.pop(next(k for k in kp if k != next(iter(kp))))  # keep the first entry and one more
        dx, dy = lib.derivatives2(bw_acc[ref])
        st = lib.gauss_filter(lib.structure_tensor(dx, dy), lib.gauss_taps(p.sigma_structure_tensor))
        kp[kkey] = lib.kernel_param(st, p)
    kparam = kp[kkey]
    fc = keep.setdefault("tail_flow", {})
    mc = keep.setdefault("tail_mask", {})
    sc = keep.setdefault("tail_sums", {})
    if "ref_half" not in keep:
        keep["ref_half"] = lib.debayer_subsample(burst.raw[ref], burst.cfa, max_val)
    ref_half = keep["ref_half"]
    acc = np.zeros((Ho, Wo, 3), lib.dtype)
    wsum = np.zeros((Ho, Wo, 3), lib.dtype)
    for i in [ref] + [k for k in range(n) if k != ref]:
        ti = None if i == ref else np.asarray(tiles[i])
        if i in sc and sc[i][0] == mkey and sc[i][1] == kkey and (i == ref or np.array_equal(sc[i][2], ti)):
            a_i, w_i = sc[i][3], sc[i][4]
        else:
            a_i = np.zeros((Ho, Wo, 3), lib.dtype)
            w_i = np.zeros((Ho, Wo, 3), lib.dtype)
            if i == ref:
                lib.accumulate(burst.raw[ref], burst.cfa, a_i, w_i, np.ones((H // 2, W // 2, 4), lib.dtype), kparam,
                               np.zeros((H, W, 2), lib.dtype), white, black, s, origin, crop, bilinear=bil)
            else:
                if i in fc and np.array_equal(fc[i][0], ti):
                    flow = fc[i][1]
                else:
                    flow = lib.flow_from_tiles(lib.arr(ti), W, H, pre.shift(ref, i), pre.rotation(ref, i), p.levels[0].tile_size)
                    for _ in range(p.iterations_lk):
                        warped = lib.warp(bw_acc[i], flow)
                        ix, iy, it = lib.derivatives(warped, bw_acc[ref])
                        flow = lib.lucas_kanade(flow, ix, iy, it, p.window_size_lk // 2, p.f32("min_det_lk"))
                    fc.setdefault(i, (ti.copy(), flow))
                if i in mc and mc[i][0] == mkey and np.array_equal(mc[i][1], ti):
                    eroded = mc[i][2]
                else:
                    mov_half = lib.debayer_subsample(burst.raw[i], burst.cfa, max_val)
                    mask = lib.robustness_mask(ref_half, mov_half, flow, float(np.float32(burst.noise_a)), float(np.float32(burst.noise_b)),
                                               p.f32("threshold_m"), np.ones((H // 2, W // 2, 4), lib.dtype), mkey[0], mkey[1], bilinear=bil)
                    eroded = lib.erode(mask, p.erode_size)
                    mc.setdefault(i, (mkey, ti.copy(), eroded))
                lib.accumulate(burst.raw[i], burst.cfa, a_i, w_i, lib.arr(eroded), kparam, lib.arr(flow), white, black, s, origin, crop,
                               bilinear=bil)
            sc.setdefault(i, (mkey, kkey, None if ti is None else ti.copy(), a_i, w_i))
        acc += a_i
        wsum += w_i
    image = lib.apply_weighting(np.zeros((Ho, Wo, 3), lib.dtype), acc, wsum, thr)
    return MergeResult(image=image, acc=acc, wsum=wsum)


def accumulate_canvas_ref(lib, raw, cfa, acc, wsum, mask, kp4, flow, white, black, s):
    """Full-frame 2x merge with the reference's central-crop kernel
    (accumulateImagesSuperRes, DeBayerKernels.cu:379-468): the frame is
    embedded in a canvas twice its size so that the canvas's central crop is
    the whole frame; kernel parameters and flow are edge-padded (the clamp /
    mirror texture reads at the frame edge), raw and mask are zero-padded
    (never read outside the crop). Requires s == 2 and W, H divisible by 4."""
    if s != 2.0:
        raise ValueError("the reference kernel only merges at 2x")
    H, W = raw.shape
    if W % 4 or H % 4:
        raise ValueError("canvas embedding needs W and H divisible by 4")
    ox, oy = W // 2, H // 2
    canvas_raw = np.zeros((2 * H, 2 * W), np.uint16)
    canvas_raw[oy:oy + H, ox:ox + W] = raw
    kpc = np.pad(kp4, ((oy, oy), (ox, ox), (0, 0)), mode="edge")
    flc = np.pad(flow, ((oy, oy), (ox, ox), (0, 0)), mode="edge")
    mc = np.zeros((H, W, 4), lib.dtype)
    mc[oy // 2:oy // 2 + H // 2, ox // 2:ox // 2 + W // 2] = mask
    lib.accumulate_ref(canvas_raw, cfa, acc, wsum, mc, kpc, flc, white, black, True)


# ---- global pre-alignment (checker) -------------------------------------------
# PreAlignment.ScanAngles (PEFStudioDX/PreAlignment.cs:176-261) and
# PreAlignmentStore (PEFStudioDX/PreAlignmentStore.cs:36-110), in FP64. The
# reference rotates with NPP WarpAffine (InterpolationMode.Cubic); NPP's cubic
# kernel and pixel-centre convention are not published, so this restatement
# defines them: Keys' cubic convolution (a = -0.5) on a 4 x 4 neighbourhood with
# clamped taps, integer pixel centres, rotation about (W/2, H/2) as
# Matrix3x3.RotAroundCenter (Matrix.cs:93-99) composes it, destination pixels
# whose source falls outside the frame left at 0 (the Set(0) before the warp).

def _keys(t, a=-0.5):
    t = np.abs(t)
    return np.where(t <= 1, ((a + 2) * t - (a + 3)) * t * t + 1,
                    np.where(t < 2, ((a * t - 5 * a) * t + 8 * a) * t - 4 * a, 0.0))


def rotate_cubic(img, angle_deg):
    H, W = img.shape
    r = angle_deg / 180.0 * np.pi
    ca, sa = np.cos(r), np.sin(r)
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    dx, dy = x - W / 2.0, y - H / 2.0
    sx, sy = ca * dx - sa * dy + W / 2.0, sa * dx + ca * dy + H / 2.0
    inside = (sx >= 0) & (sx <= W - 1) & (sy >= 0) & (sy <= H - 1)
    x0, y0 = np.floor(sx), np.floor(sy)
    ax, ay = sx - x0, sy - y0
    x0, y0 = x0.astype(np.int64), y0.astype(np.int64)
    out = np.zeros((H, W))
    for j in range(4):
        wy = _keys(ay - (j - 1))
        yy = np.clip(y0 - 1 + j, 0, H - 1)
        row = np.zeros((H, W))
        for i in range(4):
            xx = np.clip(x0 - 1 + i, 0, W - 1)
            row += _keys(ax - (i - 1)) * img[yy, xx]
        out += wy * row
    return np.where(inside, out, 0.0)


def scan_angles(ref_img, img, incr, rng, zero):
    """(x, y, angle, value) of `img` against `ref_img` (PreAlignment.cs:176-261)."""
    H, W = img.shape
    R = np.fft.rfft2(ref_img)
    max_val, max_ang, max_x, max_y = -np.finfo(np.float64).max, 0.0, 0, 0
    for phase in range(2):
        step = 5 * incr if phase == 0 else incr
        ang = zero - rng
        while ang <= zero + rng:
            T = np.fft.rfft2(rotate_cubic(img, ang))
            cc = np.fft.irfft2(np.conj(R) * T, s=(H, W))
            k = int(np.argmax(cc))
            v = cc.flat[k]  # numpy's inverse already divides by W * H, as the reference's Div after cuFFT does
            if v > max_val:
                max_val, max_ang, max_x, max_y = v, ang, k % W, k // W
            ang += step
        zero, rng = max_ang, 10 * incr
    if max_x > W // 2:
        max_x -= W
    if max_y > H // 2:
        max_y -= H
    return (-float(max_x), -float(max_y), max_ang, max_val)


def prealign_store(init):
    """PreAlignmentStore constructor: shifts (n x 2), rotations (n), reference index."""
    n = len(init)
    basic = [(0.0, 0.0, 0.0)] * n
    for i in range(1, n):
        basic[i - 1] = (init[i][0] - init[i - 1][0], init[i][1] - init[i - 1][1], init[i][2] - init[i - 1][2])
    min_index, min_shift = -1, np.finfo(np.float64).max
    for i in range(n - 1):
        ax = ay = 0.0
        for j in range(i):
            ax -= basic[j][0]; ay -= basic[j][1]
        bx = by = 0.0
        for j in range(i, n - 1):
            bx += basic[j][0]; by += basic[j][1]
        d = np.sqrt((ax + bx) ** 2 + (ay + by) ** 2)
        if d < min_shift:
            min_shift, min_index = d, i
    shifts = np.zeros((n, 2), np.float32)
    rots = np.zeros(n, np.float32)
    for i in range(n):
        a = [0.0, 0.0, 0.0]
        for j in range(i, min_index):
            for c in range(3):
                a[c] -= basic[j][c]
        for j in range(min_index, i):
            for c in range(3):
                a[c] += basic[j][c]
        shifts[i] = (a[0], a[1])
        rots[i] = a[2]
    return shifts, rots, min_index


def prealign_images(images, incr=float(np.float32(0.1)), rng=float(np.float32(1.0)), rolls=None):
    """ComputePreAlignment (controller :1451-1528) on tracking images n x H x W."""
    n = len(images)
    init = [(0.0, 0.0, 0.0, 0.0)] * n
    r0 = -float(rolls[0]) if rolls is not None else 0.0
    for i in range(1, n):
        rt = -float(rolls[i]) if rolls is not None else 0.0
        zero = float(np.float32(rt) - np.float32(r0))
        init[i] = scan_angles(images[0], images[i], incr, rng, zero)
    return init, prealign_store(init)
