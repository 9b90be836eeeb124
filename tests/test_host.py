"""Host-side logic and the C ABI surface (no GPU calls): exported symbols,
parameter defaults, output geometry, tracking-strategy bookkeeping, argument
checks."""
import ctypes
import os
import re

import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "isa.h")).read()
    return sorted(set(re.findall(r"^ISA_API\s+[\w\s\*]+?\b(isa_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = isa.lib()
    decl = header_symbols()
    assert len(decl) >= 30
    for name in decl:
        assert hasattr(lib, name), name
    assert sorted(isa.EXPORTS) == decl


def test_exported_symbols_are_sm100a_library():
    assert isa.lib().isa_version().decode().endswith("(sm_100a)")


def test_param_defaults_match_reference_defaults():
    c = isa.IsaParams()
    isa.lib().isa_params_default(ctypes.byref(c))
    p = P.MergeParams()
    for name in ("sigma_debayer_tracking", "sigma_debayer_accumulation", "high_pass", "high_pass_sigma", "matching_threshold",
                 "sigma_structure_tensor", "dth", "dtr", "k_detail", "k_denoise", "k_stretch", "k_shrink", "min_det_lk", "threshold_m",
                 "robust_s", "robust_t"):
        assert getattr(c, name) == pytest.approx(np.float32(getattr(p, name))), name
    for name in ("clear_axis", "iterations_lk", "window_size_lk", "erode_size", "tracking_strategy", "tracking_block_size"):
        assert getattr(c, name) == getattr(p, name), name
    assert c.level_count == 4
    assert [(c.levels[i].resize_level, c.levels[i].tile_size, c.levels[i].max_shift) for i in range(4)] == \
           [(1, 32, 2), (2, 32, 4), (4, 32, 4), (8, 32, 4)]
    assert c.fused_accumulate == 1 and c.super_resolution == 0 and c.merge_scale == 0


@pytest.mark.parametrize("mode,expect", [("plain", (6016, 4000)), ("super", (6016, 4000)), ("x2", (12032, 8000)), ("x1.5", (9024, 6000))])
def test_output_geometry(mode, expect):
    p = P.MergeParams()
    if mode == "super":
        p.super_resolution = True
    elif mode == "x2":
        p.merge_scale = 2.0
    elif mode == "x1.5":
        p.merge_scale = 1.5
    assert isa.output_size(isa.make_params(p), 6016, 4000) == expect


@pytest.mark.parametrize("strategy", [P.FULL, P.ONLY_ON_REFERENCE, P.ON_REFERENCE_BLOCK, P.BLOCKS])
def test_strategy_tables_match_reference_bookkeeping(strategy):
    for n in (2, 3, 5, 8, 20, 33):
        for ref in sorted({0, n // 2, n - 1}):
            for blk in (1, 2, 3, 5, 40):
                pairs, rows = isa.tracking_pairs(n, ref, strategy, blk)
                assert pairs.shape[0] == P.shift_count(n, strategy, P.effective_block(n, blk))
                np.testing.assert_array_equal(pairs, np.array(P.shift_pairs(n, ref, strategy, blk)).reshape(-1, 2))
                A = P.shift_matrix(n, ref, strategy, blk)
                B = np.zeros_like(A)
                for k, (a, b, sg) in enumerate(rows):
                    B[k, a:b] = sg
                np.testing.assert_array_equal(A, B)
                idx = P.index_table(n, ref, strategy, blk)
                # every tracked pair has its own measurement row
                rows_of_pairs = sorted(idx[r, t] for r, t in pairs)
                assert rows_of_pairs == list(range(len(pairs)))


def test_full_strategy_counts():
    assert P.shift_count(20, P.FULL, 5) == 190
    assert P.shift_count(50, P.FULL, 5) == 1225
    assert P.shift_count(8, P.FULL, 5) == 28


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = isa.lib()
    ctx = ctypes.c_void_p()
    good = isa.make_params()
    assert lib.isa_ctx_create(ctypes.byref(ctx), 15, 16, 4, ctypes.byref(good)) == isa.ISA_EINVAL
    assert lib.isa_ctx_create(ctypes.byref(ctx), 64, 64, 1, ctypes.byref(good)) == isa.ISA_EINVAL
    bad = isa.make_params()
    bad.levels[1].tile_size = 31  # odd tiles are not supported (the box filter of kernel.cu:59-128 needs T even)
    assert lib.isa_ctx_create(ctypes.byref(ctx), 512, 512, 4, ctypes.byref(bad)) == isa.ISA_EINVAL
    assert b"invalid" in lib.isa_last_error()
    bad = isa.make_params()
    bad.levels[0].resize_level = 2
    assert lib.isa_ctx_create(ctypes.byref(ctx), 512, 512, 4, ctypes.byref(bad)) == isa.ISA_EINVAL
    bad = isa.make_params()
    bad.window_size_lk = 41
    assert lib.isa_ctx_create(ctypes.byref(ctx), 512, 512, 4, ctypes.byref(bad)) == isa.ISA_EINVAL
    assert lib.isa_tracking_pairs(5, 7, 0, 5, None, None, 0) == isa.ISA_EINVAL
    assert lib.isa_tracking_pairs(5, 0, 9, 5, None, None, 0) == isa.ISA_EINVAL
    cfa = (ctypes.c_int * 4)(0, 1, 1, 3)
    f3 = (ctypes.c_float * 3)(1, 1, 1)
    assert lib.isa_debayer_full(ctypes.c_void_p(16), ctypes.c_size_t(128), 64, 64, cfa, f3, f3, f3, ctypes.c_void_p(16),
                                ctypes.c_size_t(768), None) == isa.ISA_EINVAL


def test_gauss_taps_follow_controller_rule(oracle):
    # gaussian_filter_1D: size = (int)(sigma/0.6 - 0.4)*2 + 3
    assert len(oracle.gauss_taps(0.5)) == 3
    assert len(oracle.gauss_taps(1.0)) == 5
    assert len(oracle.gauss_taps(2.0)) == 7
    assert len(oracle.gauss_taps(0.0)) == 9 and oracle.gauss_taps(0.0)[4] == 1
    assert abs(oracle.gauss_taps(1.0).sum() - 1) < 1e-12


def test_dng_decode_halves_and_file_handles_check_their_arguments():
    """isa_dng_decode_begin / _finish, isa_dng_roll_angle, isa_dng_file_info and
    isa_pef_file_info refuse NULL and bad layouts before any CUDA call."""
    lib = isa.lib()
    fake = ctypes.c_void_p(256)
    L = isa.IsaDngLayout()
    for fn in (lib.isa_dng_decode_begin, lib.isa_dng_decode_finish):
        assert fn(None, fake, ctypes.c_size_t(16), ctypes.byref(L), 8, 8, fake, ctypes.c_size_t(1 << 20), fake, ctypes.c_size_t(16),
                  None) == isa.ISA_EINVAL
        assert fn(fake, fake, ctypes.c_size_t(16), ctypes.byref(L), 8, 8, fake, ctypes.c_size_t(1 << 20), fake, ctypes.c_size_t(16),
                  None) == isa.ISA_EINVAL   # n = 0: a bad layout
    # a valid uncompressed layout with an output pitch below one row: refused by both halves before any CUDA call
    offs, cnts = (ctypes.c_uint32 * 1)(0), (ctypes.c_uint32 * 1)(128)
    good = isa.IsaDngLayout(tiled=0, rows_per_strip=8, n=1, offsets=ctypes.cast(offs, ctypes.c_void_p),
                            byte_counts=ctypes.cast(cnts, ctypes.c_void_p), compression=1, bit_depth=16)
    for fn in (lib.isa_dng_decode_begin, lib.isa_dng_decode_finish):
        assert fn(fake, fake, ctypes.c_size_t(128), ctypes.byref(good), 8, 8, fake, ctypes.c_size_t(1 << 20), fake, ctypes.c_size_t(15),
                  None) == isa.ISA_EINVAL
        assert b"output pitch" in lib.isa_last_error()
    roll = ctypes.c_float()
    assert lib.isa_dng_roll_angle(None, ctypes.byref(roll)) == isa.ISA_EINVAL
    assert lib.isa_dng_file_info(None, None, None, None, None, None) == isa.ISA_EINVAL
    assert lib.isa_pef_file_info(None, None) == isa.ISA_EINVAL
    h = ctypes.c_void_p()
    assert lib.isa_dng_open(None, ctypes.c_size_t(0), ctypes.byref(h)) == isa.ISA_EINVAL
    assert lib.isa_pef_open(ctypes.c_char_p(b"II*\0"), ctypes.c_size_t(4), ctypes.byref(h)) == isa.ISA_EINVAL
    assert lib.isa_dng_close(None) == isa.ISA_OK and lib.isa_pef_close(None) == isa.ISA_OK
