"""Seeded per-kernel cases shared by the golden-vector generator and the tests.

run_all(lib) runs every case through a checker StageLib (oracle/pipeline.py)
and returns {name: array}; inputs are recorded as `in_*`, outputs as `out_*`.
Generated with the reference's own kernels (ref64), re-run with the FP64
restatement (oracle64) by tests/test_oracle_golden.py.
"""
from __future__ import annotations

import numpy as np

from imagestackalignator_b200 import params as P


def _raw(rng, W, H, lo=512, hi=16383):
    # smooth structure + noise so demosaic gradients are non-trivial
    y, x = np.mgrid[0:H, 0:W]
    base = 0.4 + 0.25 * np.sin(x / 5.0) * np.cos(y / 7.0) + 0.1 * (x > W // 2)
    img = base + rng.normal(0, 0.02, (H, W))
    return np.clip(lo + img * (hi - lo), 0, 16383).astype(np.uint16)


def _img(rng, W, H):
    y, x = np.mgrid[0:H, 0:W]
    return (0.5 + 0.2 * np.sin(x / 3.0 + y / 5.0) + 0.15 * np.cos(x / 11.0) * np.sin(y / 4.0) + rng.normal(0, 0.01, (H, W)))


def run_all(lib):
    rng = np.random.default_rng(20261203)
    out = {}
    # A1 demosaic, two CFA layouts
    for name, cfa in (("rggb", (0, 1, 1, 2)), ("grbg", (1, 0, 2, 1))):
        raw = _raw(rng, 48, 40)
        out[f"in_raw_{name}"] = raw
        out[f"out_debayer_{name}"] = lib.debayer_full(raw, cfa, (512.0, 500.0, 520.0), np.float32([1.0, 1.0 / 1.5, 1.0 / 2.0]),
                                                      np.float32([15871.0, 15871.0 / 1.5, 15871.0 / 2.0]))
    # A2 gamma and the Fourier filter coefficients
    rgb = rng.uniform(-0.1, 1.1, (24, 32, 3))
    rgb[0, 0, 0] = np.nan
    out["in_gamma"] = rgb
    out["out_gamma"] = lib.gamma_srgb(rgb)
    out["out_fourier_96x64"] = lib.fourier_mask(96, 64, 1.0, float(np.float32(0.01)), 1.0, float(np.float32(0.0025)), 0)
    out["out_fourier_clear"] = lib.fourier_mask(64, 48, 1.0, 0.05, 1.0, 0.02, 3)
    out["out_fourier_lowpass"] = lib.fourier_mask(64, 48, 0.3, 0.0, 0.05, 0.0, 0)
    # A3 tile tracking: known structure, search shifted by a few pixels
    for S in (2, 4):
        W, H, T = 168, 136, 32
        ref = _img(rng, W, H)
        trk = np.roll(ref, (1, -2), axis=(0, 1)) + rng.normal(0, 0.003, (H, W))
        tcx, tcy = (W - 2 * S) // T, (H - 2 * S) // T
        pre = rng.uniform(-1.5, 1.5, (tcy, tcx, 2))
        out[f"in_track_ref_s{S}"] = ref
        out[f"in_track_trk_s{S}"] = trk
        out[f"in_track_pre_s{S}"] = pre
        g, sc = lib.track_pair(trk, ref, T, S, tcx, tcy, pre, (0.7, -0.3), 0.002, (-0.4, 0.9), -0.001, 1.0, want_scores=True)
        out[f"out_track_s{S}"] = g
        out[f"out_scores_s{S}"] = sc
    # A4 upsampling
    grid = rng.uniform(-3, 3, (5, 7, 2))
    out["in_upsample"] = grid
    out["out_upsample"] = lib.upsample_shifts(grid, 4, 2, 13, 10, 32, 32)
    # A5 solve (Full with outliers, OnlyOnReference) and optimal shifts
    for name, strat, n, ref in (("full", P.FULL, 6, 0), ("onref", P.ONLY_ON_REFERENCE, 5, 2), ("blocks", P.BLOCKS, 6, 0)):
        A = P.shift_matrix(n, ref, strat, 3)
        truth = rng.uniform(-4, 4, (12, n - 1, 2))
        meas = np.einsum("mk,tkc->tmc", A, truth) + rng.normal(0, 0.05, (12, A.shape[0], 2))
        meas[::3, 0, :] += 7.0  # outliers
        out[f"in_solve_{name}"] = meas
        m2, x, st = lib.solve_shifts(A, meas)
        out[f"out_solve_meas_{name}"] = m2
        out[f"out_solve_x_{name}"] = x
        out[f"out_solve_status_{name}"] = st.astype(np.int64)
        out[f"out_optimal_{name}"] = lib.optimal_shifts(x, 4, 3, ref, n - 1)
    # A6 flow, warp, derivatives, LK
    W, H = 64, 48
    tiles = rng.uniform(-2, 2, (4, 5, 2))
    out["in_tiles"] = tiles
    flow = lib.flow_from_tiles(tiles, W, H, (1.25, -0.5), 0.003, 12)
    out["out_flow"] = flow
    src, tgt = _img(rng, W, H), _img(rng, W, H)
    out["in_src"], out["in_tgt"] = src, tgt
    out["out_warp"] = lib.warp(src, flow)
    ix, iy, it = lib.derivatives(out["out_warp"], tgt)
    out["out_ix"], out["out_iy"], out["out_it"] = ix, iy, it
    dx, dy = lib.derivatives2(src)
    out["out_dx"], out["out_dy"] = dx, dy
    out["out_lk"] = lib.lucas_kanade(flow, ix, iy, it, 5, float(np.float32(0.01)))
    # A7 subsample, robustness mask
    raw = _raw(rng, 64, 48)
    raw2 = np.roll(raw, (2, 4), axis=(0, 1))
    out["in_raw_mask_ref"], out["in_raw_mask_mov"] = raw, raw2
    h1 = lib.debayer_subsample(raw, (0, 1, 1, 2), 16383.0)
    h2 = lib.debayer_subsample(raw2, (0, 1, 1, 2), 16383.0)
    out["out_half_ref"], out["out_half_mov"] = h1, h2
    fl = rng.uniform(-3, 3, (48, 64, 2))
    out["in_mask_flow"] = fl
    ones = np.ones((24, 32, 4))
    out["out_mask"] = lib.robustness_mask(h1, h2, fl, float(np.float32(4e-4)), float(np.float32(2e-6)), 100000.0, ones)
    out["out_mask_m"] = lib.robustness_mask(h1, h2, fl, float(np.float32(4e-4)), float(np.float32(2e-6)), 1e-4, ones)
    # A8 structure tensor and kernel parameters
    st = lib.structure_tensor(dx, dy)
    out["out_st"] = st
    out["out_kparam"] = lib.kernel_param(st, P.MergeParams())
    # A9 accumulation: plain and super-resolution reference kernels
    W, H = 64, 48
    raw = _raw(rng, W, H)
    out["in_acc_raw"] = raw
    kp = lib.kernel_param(lib.structure_tensor(*lib.derivatives2(_img(rng, W, H) * 0.3)), P.MergeParams())
    kp[3, 5] = np.nan  # exercises the non-finite weight rule
    out["in_acc_kparam"] = kp
    fl = rng.uniform(-2.5, 2.5, (H, W, 2))
    out["in_acc_flow"] = fl
    mk = rng.uniform(0, 1, (H // 2, W // 2, 4))
    mk[2, 3, 1] = np.nan
    out["in_acc_mask"] = mk
    white, black = (15871.0, 15871.0, 15871.0), (512.0, 512.0, 512.0)
    acc = np.zeros((H, W, 3), lib.dtype)
    wsum = np.zeros((H, W, 3), lib.dtype)
    if lib.pfx == "ref_":
        lib.accumulate_ref(raw, (0, 1, 1, 2), acc, wsum, mk, kp, fl, white, black, False)
    else:
        lib.accumulate(raw, (0, 1, 1, 2), acc, wsum, mk, kp, fl, white, black, 1.0, (0, 0), (0, 0, W - 1, H - 1))
    out["out_acc_plain"], out["out_wsum_plain"] = acc.copy(), wsum.copy()
    kp4 = np.concatenate([kp, np.zeros((H, W, 1))], axis=2)
    acc[:] = 0
    wsum[:] = 0
    if lib.pfx == "ref_":
        lib.accumulate_ref(raw, (0, 1, 1, 2), acc, wsum, mk, kp4, fl, white, black, True)
    else:
        lib.accumulate(raw, (0, 1, 1, 2), acc, wsum, mk, kp, fl, white, black, 2.0, (W // 2, H // 2),
                       (W // 4, H // 4, W // 2 - 1 + W // 4, H // 2 - 1 + H // 4))
    out["out_acc_super"], out["out_wsum_super"] = acc.copy(), wsum.copy()
    # whole-frame 2x: the reference kernel on a canvas twice the frame size
    import pipeline as PL
    acc2 = np.zeros((2 * H, 2 * W, 3), lib.dtype)
    wsum2 = np.zeros((2 * H, 2 * W, 3), lib.dtype)
    if lib.pfx == "ref_":
        PL.accumulate_canvas_ref(lib, raw, (0, 1, 1, 2), acc2, wsum2, mk, kp4, fl, white, black, 2.0)
    else:
        lib.accumulate(raw, (0, 1, 1, 2), acc2, wsum2, mk, kp, fl, white, black, 2.0, (0, 0), (0, 0, W - 1, H - 1))
    out["out_acc_full2x"], out["out_wsum_full2x"] = acc2, wsum2
    # A10 finalize
    dec = rng.uniform(0, 1, (H, W, 3))
    out["in_dec"] = dec
    out["out_weight_plain"] = lib.apply_weighting(dec, out["out_acc_plain"], out["out_wsum_plain"], 1.0)
    out["out_weight_super"] = lib.apply_weighting(dec, out["out_acc_super"], out["out_wsum_super"], 0.0)
    return out
