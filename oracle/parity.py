"""Decision-aware parity of a merged burst -- TEST INFRASTRUCTURE ONLY.

The merged image depends on the dense flows only through rounded values:
the accumulation's shift round(s * flow) (DeBayerKernels.cu:310-311,
403-404) and the robustness mask's moved-pixel offset round(flow / 2)
(RobustnessModell.cu:401-402, sampled at the half-resolution pixel), plus
ApplyWeighting's test w < threshold (kernel.cu:336-391). Where such a
decision differs between the GPU and the FP64 oracle (a value within FP32
noise of a half-integer, or an ill-conditioned LK window that moved a flow
across one), the output pixel may differ by up to the local contrast; every
other pixel must agree to 1e-4 of the white level (the whole-path bar).

`merge_parity` finds those decisions from both sides' flows, masks and
weight sums, excludes exactly the output pixels that read a differing
decision, checks that every mask value that differs is explained by a
differing rounding decision, and asserts max |GPU - FP64| <= 1e-4 over the
rest. Given the oracle's accumulation fed the GPU's own flows, masks and
kernel parameters, it also holds the accumulation to the bar on every pixel,
and counts the pixels whose difference from the pure oracle is carried in
from those FP32 inputs (the kernel's orientation is ill-conditioned where
the structure tensor is nearly isotropic). `track_parity` compares the integer tile shifts (the first minimum of
every tile's L2 map, kernel.cu:422-546) of every pair at every pyramid level.

Only the tests and the smoke check import this module.
"""
from __future__ import annotations

import numpy as np

IMAGE_BAR = 1e-4      # max |GPU - FP64| in units of the white level, over decision-matched pixels
MASK_DECISION = 1e-5  # an eroded-mask value differing by more than this was decided differently
TIE_MARGIN = 1e-5     # relative L2 margin under which two shifts of a tile tie at FP32 resolution


def c_round(v):
    """C round(): half away from zero."""
    return np.where(v >= 0, np.floor(v + 0.5), -np.floor(-v + 0.5))


def near_half(v, margin):
    """v within `margin` (scalar, or per point for the last axis of v) of a half-integer."""
    f = np.abs(v) - np.floor(np.abs(v))
    margin = np.asarray(margin)
    if margin.ndim and margin.ndim < np.ndim(v):
        margin = margin[..., None]
    return np.abs(f - 0.5) < margin


def mirror_index(i, n):
    p = 2 * n
    j = np.mod(i, p)
    return np.where(j >= n, p - 1 - j, j)


def bilinear(img, xb, yb, mirror):
    """The oracle's texture sampler (isa_oracle.c `bilinear`), vectorised:
    img H x W x C, sample points xb, yb (texel units, centre at integer)."""
    H, W = img.shape[:2]
    fx, fy = np.floor(xb), np.floor(yb)
    i, j = fx.astype(np.int64), fy.astype(np.int64)
    a, b = xb - fx, yb - fy
    if mirror:
        i0, i1, j0, j1 = mirror_index(i, W), mirror_index(i + 1, W), mirror_index(j, H), mirror_index(j + 1, H)
    else:
        i0, i1 = np.clip(i, 0, W - 1), np.clip(i + 1, 0, W - 1)
        j0, j1 = np.clip(j, 0, H - 1), np.clip(j + 1, 0, H - 1)
    a = a[..., None]
    b = b[..., None]
    img = np.asarray(img, np.float64)
    v = np.where((a != 1) & (b != 1), (1 - a) * (1 - b) * img[j0, i0], 0.0)
    v = v + np.where((a != 0) & (b != 1), a * (1 - b) * img[j0, i1], 0.0)
    v = v + np.where((a != 1) & (b != 0), (1 - a) * b * img[j1, i0], 0.0)
    v = v + np.where((a != 0) & (b != 0), a * b * img[j1, i1], 0.0)
    return v


def bilinear_f32(img, xb, yb, mirror):
    """The GPU kernels' FP32 bilinear sample (isa::lerp2, zero-weight texels
    skipped) at FP32 positions xb, yb, evaluated in float32 without fused
    multiply-adds; returns float64."""
    f = np.float32
    xb = np.asarray(xb, f)
    yb = np.asarray(yb, f)
    H, W = img.shape[:2]
    fx, fy = np.floor(xb), np.floor(yb)
    i, j = fx.astype(np.int64), fy.astype(np.int64)
    a, b = (xb - fx).astype(f), (yb - fy).astype(f)
    if mirror:
        i0, i1, j0, j1 = mirror_index(i, W), mirror_index(i + 1, W), mirror_index(j, H), mirror_index(j + 1, H)
    else:
        i0, i1 = np.clip(i, 0, W - 1), np.clip(i + 1, 0, W - 1)
        j0, j1 = np.clip(j, 0, H - 1), np.clip(j + 1, 0, H - 1)
    img = np.asarray(img, f)
    a, b = a[..., None], b[..., None]
    one = f(1)
    v = ((one - a) * (one - b)) * img[j0, i0]
    v = np.where(a != 0, v + (a * (one - b)) * img[j0, i1], v)
    v = np.where(b != 0, v + ((one - a) * b) * img[j1, i0], v)
    v = np.where((a != 0) & (b != 0), v + (a * b) * img[j1, i1], v)
    return v.astype(np.float64)


def f32_margin(v):
    """Room for the kernels' fused multiply-adds in an FP32 value v: a few ulps."""
    return 1e-6 + 8.0 * np.abs(v) * 2.0 ** -24


def dilate(mask2d, r):
    """Binary dilation by a (2r+1) x (2r+1) square with the border replicated."""
    if r <= 0:
        return mask2d.copy()
    H, W = mask2d.shape
    p = np.pad(mask2d, r, mode="edge")
    out = np.zeros_like(mask2d)
    for dy in range(2 * r + 1):
        for dx in range(2 * r + 1):
            out |= p[dy:dy + H, dx:dx + W]
    return out


def gpu_shift_values(flow, x, y, s, origin):
    """s * flow as the accumulation kernels compute it in FP32 at output pixel
    (x, y): position ((float)x + 0.5f + ox) / s - 0.5f, FP32 bilinear, times s."""
    f = np.float32
    gx = ((x.astype(f) + f(0.5) + f(origin[0])) / f(s) - f(0.5)).astype(f)
    gy = ((y.astype(f) + f(0.5) + f(origin[1])) / f(s) - f(0.5)).astype(f)
    return (bilinear_f32(flow, gx, gy, True).astype(f) * f(s)).astype(np.float64)


def _out_coords(Wo, Ho, s, origin):
    y, x = np.mgrid[0:Ho, 0:Wo].astype(np.float64)
    xb = (x + 0.5 + origin[0]) / s - 0.5
    yb = (y + 0.5 + origin[1]) / s - 0.5
    return x, y, xb, yb


def merge_parity(got, want, flows_gpu, flows_orc, masks_gpu, masks_orc, geometry, erode_size, wsum_orc=None, ref=0,
                 max_excluded=0.02, bar=IMAGE_BAR, maps=None, wsum_gpu=None, want_sub=None, wsum_sub=None):
    """got / want: Ho x Wo x 3 merged images (GPU, FP64 oracle). flows_*: dict
    frame -> H x W x 2; masks_*: dict frame -> H/2 x W/2 x 4 (eroded).
    geometry: (Wo, Ho, s, origin, crop, thr) as oracle/pipeline.out_geometry.
    wsum_gpu / wsum_orc: Ho x Wo x 3 weight sums; ApplyWeighting's decision
    w < thr is compared between them (with only wsum_orc, oracle sums within
    a relative 1e-4 of thr count as undecided). want_sub (optional): the
    oracle's accumulation and ApplyWeighting (pipeline.merge_tail) fed the
    GPU's flows, masks and kernel parameters; it must match the GPU to the bar on every pixel
    whose shift the GPU's FP32 interpolation cannot round either way, and a
    pixel where it matches while the pure oracle does not is counted as
    carried in from upstream FP32 inputs instead of failing. wsum_sub: its
    weight sums, for its own ApplyWeighting decision.
    Returns a dict of counts; raises AssertionError when the bar fails.
    maps (a dict, optional) receives the per-pixel |difference| and the
    excluded-pixel masks before the bar is checked."""
    Wo, Ho, s, origin, crop, thr = geometry
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape == (Ho, Wo, 3), (got.shape, want.shape)
    assert np.isfinite(got).all(), "non-finite values in the merged image"
    x, y, xb, yb = _out_coords(Wo, Ho, s, origin)
    excl_shift = np.zeros((Ho, Wo), bool)
    excl_mask = np.zeros((Ho, Wo), bool)
    stats = {"frames": 0, "shift_decisions_differ": 0, "mask_cells_differ": 0, "mask_cells_unexplained": 0}
    exact_s = float(s) == 1.0 and tuple(origin) == (0, 0)
    # mask cells read by each output pixel: ux // 2 for the 25 unshifted taps
    ux = [np.clip(np.floor((x + px + origin[0]) / s), crop[0], crop[2]).astype(np.int64) // 2 for px in range(-2, 3)]
    uy = [np.clip(np.floor((y + py + origin[1]) / s), crop[1], crop[3]).astype(np.int64) // 2 for py in range(-2, 3)]
    for i in sorted(flows_gpu):
        if i == ref:
            continue
        stats["frames"] += 1
        fg, fo = np.asarray(flows_gpu[i], np.float64), np.asarray(flows_orc[i], np.float64)
        H, W = fg.shape[:2]
        # accumulation shift at each output pixel: the GPU's own FP32 sample (DeBayerKernels.cu:403-404 positions)
        vg = gpu_shift_values(fg, x, y, s, origin)
        vo = bilinear(fo, xb, yb, True) * s
        d = (c_round(vg) != c_round(vo)).any(axis=2)
        if not exact_s:
            d |= near_half(vg, f32_margin(vg)).any(axis=2)
        d[[0, -1], :] = False
        d[:, [0, -1]] = False
        stats["shift_decisions_differ"] += int(d.sum())
        excl_shift |= d
        # robustness-mask offsets round(flow / 2) at each half-resolution pixel, and the eroded masks
        Hh, Wh = H // 2, W // 2
        hy, hx = np.mgrid[0:Hh, 0:Wh].astype(np.float64)
        cxb, cyb = (hx + 0.5) / Wh * W - 0.5, (hy + 0.5) / Hh * H - 0.5
        # the robustness kernel's position ((float)x + 0.5f) / Wh * Wf - 0.5f, rounded after the product or fused
        # with the subtraction: a cell whose offset depends on which is undecided
        f = np.float32
        qx, qy = ((hx.astype(f) + f(0.5)) / f(Wh)).astype(f), ((hy.astype(f) + f(0.5)) / f(Hh)).astype(f)
        hgs = []
        for fused in (False, True):
            if fused:
                gxb, gyb = (qx.astype(np.float64) * W - 0.5).astype(f), (qy.astype(np.float64) * H - 0.5).astype(f)
            else:
                gxb, gyb = ((qx * f(W)).astype(f) - f(0.5)).astype(f), ((qy * f(H)).astype(f) - f(0.5)).astype(f)
            hgs.append((bilinear_f32(fg, gxb, gyb, True).astype(f) * f(0.5)).astype(np.float64))
        hg = hgs[0]
        ho = bilinear(fo, cxb, cyb, True) * 0.5
        md = (c_round(hg) != c_round(ho)).any(axis=2) | (c_round(hgs[1]) != c_round(ho)).any(axis=2)
        md |= near_half(hg, f32_margin(hg)).any(axis=2) | near_half(hgs[1], f32_margin(hgs[1])).any(axis=2)
        mg, mo = np.asarray(masks_gpu[i], np.float64), np.asarray(masks_orc[i], np.float64)
        mdiff = (np.abs(mg - mo)[..., :3] > MASK_DECISION).any(axis=2)
        # the erosion spreads a cell's decision over erode_size x erode_size cells; the mask's
        # 3 x 3 statistics read their own cell's offset only
        explained = dilate(md, erode_size // 2)
        unexplained = mdiff & ~explained
        stats["mask_cells_differ"] += int(mdiff.sum())
        stats["mask_cells_unexplained"] += int(unexplained.sum())
        if unexplained.any():
            yy, xx = np.nonzero(unexplained)
            raise AssertionError(f"frame {i}: {unexplained.sum()} eroded-mask cells differ with no differing rounding decision, "
                                 f"e.g. cell ({xx[0]}, {yy[0]}): gpu {mg[yy[0], xx[0]]} oracle {mo[yy[0], xx[0]]}")
        for cy in uy:
            for cx in ux:
                excl_mask |= mdiff[np.clip(cy, 0, Hh - 1), np.clip(cx, 0, Wh - 1)]
    excl_w = np.zeros((Ho, Wo), bool)
    if thr > 0 and wsum_orc is not None:
        wo = np.asarray(wsum_orc, np.float64)
        if wsum_gpu is not None:
            excl_w = ((np.asarray(wsum_gpu, np.float64) < thr) != (wo < thr)).any(axis=2)
        else:
            excl_w = (np.abs(wo - thr) < 1e-4 * max(thr, 1.0)).any(axis=2)
    excl = excl_shift | excl_mask | excl_w
    diff = np.abs(got - want).max(axis=2)
    # upstream conditioning: where the pure oracle disagrees but the oracle's accumulation fed the GPU's own flows,
    # masks and kernel parameters agrees, the difference is carried in from FP32 inputs. The kernel's orientation
    # comes from the structure tensor's eigenvectors (kernel.cu:628-700), which are ill-defined where the tensor is
    # nearly isotropic, while the kernel stays anisotropic (stretch / shrink); far taps' weights exp(-q / 2) then
    # move with the FP32 rounding of the tensor, and a channel reached only by far taps (scales other than 1 and 2)
    # or normalised by a tiny certainty-weighted sum carries that into the output
    excl_cond = np.zeros((Ho, Wo), bool)
    if want_sub is not None:
        dsub = np.abs(got - np.asarray(want_sub, np.float64)).max(axis=2)
        excl_cond = ~excl & (diff > bar) & (dsub <= bar)
        # the accumulation itself: same flows and masks -> the bar on every pixel but those whose shift the GPU's FP32
        # sample rounds otherwise than FP64 on the same flows (s != 1) and a flipped ApplyWeighting threshold
        tail_skip = np.zeros((Ho, Wo), bool)
        if thr > 0 and wsum_gpu is not None and wsum_sub is not None:
            tail_skip = ((np.asarray(wsum_gpu, np.float64) < thr) != (np.asarray(wsum_sub, np.float64) < thr)).any(axis=2)
        if not exact_s:
            for i in sorted(flows_gpu):
                if i != ref:
                    fgi = np.asarray(flows_gpu[i], np.float64)
                    vg = gpu_shift_values(fgi, x, y, s, origin)
                    v64 = bilinear(fgi, xb, yb, True) * s  # what the FP64 tail takes from the same flows
                    tail_skip |= near_half(vg, f32_margin(vg)).any(axis=2) | (c_round(vg) != c_round(v64)).any(axis=2)
        stats["tail_max_abs"] = float(dsub[~tail_skip].max())
        if maps is not None:
            maps.update(tail_diff=dsub, tail_skip=tail_skip)
        assert stats["tail_max_abs"] <= bar, (f"accumulation on the GPU's own flows, masks and kernel parameters differs by {stats['tail_max_abs']:.3e}", stats)
    excl |= excl_cond
    keep = ~excl
    if maps is not None:
        maps.update(diff=diff, excluded=excl, excluded_shift=excl_shift, excluded_mask=excl_mask, excluded_weight=excl_w,
                    excluded_conditioned=excl_cond)
    stats.update(pixels=int(diff.size), excluded=int(excl.sum()), excluded_shift=int(excl_shift.sum()),
                 excluded_mask=int(excl_mask.sum()), excluded_weight=int(excl_w.sum()), excluded_conditioned=int(excl_cond.sum()),
                 max_abs_matched=float(diff[keep].max()) if keep.any() else 0.0,
                 max_abs_all=float(diff.max()), above_bar_all=int((diff > bar).sum()))
    assert stats["max_abs_matched"] <= bar, (
        f"max |GPU - FP64| = {stats['max_abs_matched']:.3e} > {bar:g} over decision-matched pixels", stats)
    assert stats["excluded"] <= max_excluded * diff.size, (f"{stats['excluded']} pixels read a differing decision", stats)
    return stats


def track_parity(record, keep, pairs, levels, W, H, max_offset_flips=0.002):
    """record: the GPU's isa_debug_track_record buffer (int32); keep: the
    oracle pipeline's intermediates (scores and unrounded offsets per
    (level, ref, trk)); pairs: (m x 2) in isa_tracking_pairs order; levels:
    the pyramid (params.TrackingLevel list). Per level and pair, every tile
    whose search block lies at the same integer offset must have the
    oracle's first-minimum index, except where the oracle's best and
    second-best L2 scores are within a relative TIE_MARGIN. A block offset
    may differ only where the upstream pre-shifts round differently (counted
    and bounded). Returns counts."""
    rec = np.asarray(record, np.int64)
    m = len(pairs)
    off = 0
    stats = {"tiles": 0, "ties": 0, "argmin_checked": 0, "offset_flips": 0}
    for li, lv in enumerate(levels):
        Wl, Hl = W // lv.resize_level, H // lv.resize_level
        tcx, tcy = (Wl - 2 * lv.max_shift) // lv.tile_size, (Hl - 2 * lv.max_shift) // lv.tile_size
        nt = tcx * tcy
        am = rec[off:off + m * nt].reshape(m, nt)
        ofs = rec[off + m * nt:off + 3 * m * nt].reshape(m, nt, 2)
        off += 3 * m * nt
        for k, (r, t) in enumerate(pairs):
            sc = keep["scores"][(li, r, t)]
            uo = keep["offsets"][(li, r, t)]
            want_am = np.argmin(sc, axis=1)
            want_of = c_round(uo).astype(np.int64)
            same_block = (ofs[k] == want_of).all(axis=1)
            srt = np.sort(sc, axis=1)
            tie = (srt[:, 1] - srt[:, 0]) <= TIE_MARGIN * np.maximum(srt[:, 0], 1e-30)
            bad = same_block & ~tie & (am[k] != want_am)
            if bad.any():
                j = int(np.nonzero(bad)[0][0])
                raise AssertionError(f"level {li} pair ({r}, {t}) tile {j}: integer shift {am[k, j]} != oracle {want_am[j]} "
                                     f"(scores {srt[j, :2]})")
            stats["tiles"] += nt
            stats["ties"] += int((tie & same_block & (am[k] != want_am)).sum())
            stats["argmin_checked"] += int(same_block.sum())
            stats["offset_flips"] += int((~same_block).sum())
    assert stats["offset_flips"] <= max_offset_flips * stats["tiles"], stats
    return stats
