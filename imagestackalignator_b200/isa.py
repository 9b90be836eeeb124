"""ctypes binding of libisa.so (include/isa.h) -- the same surface a C# host
would bind with [DllImport]. Device buffers are passed as raw pointers;
torch tensors are accepted for convenience (torch is plumbing here: device
memory and streams).

There is no CPU fallback: every compute entry point runs the CUDA kernels of
libisa.so and raises if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libisa.so")

ISA_OK, ISA_EINVAL, ISA_ECUDA, ISA_ESINGULAR, ISA_ETIMEDOUT, ISA_ENOMEM = 0, -1, -2, -3, -4, -5
MAX_LEVELS = 8


class IsaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"isa error {code}: {msg}")
        self.code = code


class IsaLevel(ctypes.Structure):
    _fields_ = [("resize_level", ctypes.c_int), ("tile_size", ctypes.c_int), ("max_shift", ctypes.c_int)]


class IsaTuning(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("lk_strip_rows", ctypes.c_int), ("acc_block_x", ctypes.c_int),
                ("acc_block_y", ctypes.c_int)]


class IsaParams(ctypes.Structure):
    _fields_ = [
        ("sigma_debayer_tracking", ctypes.c_float), ("sigma_debayer_accumulation", ctypes.c_float),
        ("high_pass", ctypes.c_float), ("high_pass_sigma", ctypes.c_float), ("clear_axis", ctypes.c_int),
        ("matching_threshold", ctypes.c_float), ("sigma_structure_tensor", ctypes.c_float),
        ("dth", ctypes.c_float), ("dtr", ctypes.c_float), ("k_detail", ctypes.c_float), ("k_denoise", ctypes.c_float),
        ("k_stretch", ctypes.c_float), ("k_shrink", ctypes.c_float), ("iterations_lk", ctypes.c_int),
        ("window_size_lk", ctypes.c_int), ("erode_size", ctypes.c_int), ("min_det_lk", ctypes.c_float),
        ("threshold_m", ctypes.c_float), ("tracking_strategy", ctypes.c_int), ("tracking_block_size", ctypes.c_int),
        ("green_channel_only", ctypes.c_int), ("level_count", ctypes.c_int), ("levels", IsaLevel * MAX_LEVELS),
        ("super_resolution", ctypes.c_int), ("merge_scale", ctypes.c_float), ("robust_s", ctypes.c_float),
        ("robust_t", ctypes.c_float), ("fused_accumulate", ctypes.c_int), ("sample_mode", ctypes.c_int),
    ]


class IsaRawInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("cfa", ctypes.c_int * 4), ("black", ctypes.c_float * 3),
                ("white", ctypes.c_float * 3), ("camera_white", ctypes.c_float * 3), ("noise_alpha", ctypes.c_float),
                ("noise_beta", ctypes.c_float)]


class IsaPrealign(ctypes.Structure):
    _fields_ = [("shifts", ctypes.POINTER(ctypes.c_float)), ("rotations_deg", ctypes.POINTER(ctypes.c_float)),
                ("reference", ctypes.c_int)]


class IsaTrackPair(ctypes.Structure):
    _fields_ = [("reference", ctypes.c_int), ("to_track", ctypes.c_int), ("grid", ctypes.c_int),
                ("base_shift_ref", ctypes.c_float * 2), ("rotation_ref", ctypes.c_float),
                ("base_shift_trk", ctypes.c_float * 2), ("rotation_trk", ctypes.c_float)]


# every symbol include/isa.h declares (checked by the CPU tests)
EXPORTS = [
    "isa_params_default", "isa_last_error", "isa_version", "isa_ctx_create", "isa_ctx_destroy", "isa_output_size", "isa_stage_times",
    "isa_launch_count", "isa_tracking_pairs",
    "isa_merge_burst", "isa_merge_burst_host", "isa_debug_buffers", "isa_debug_shifts", "isa_debug_track_record",
    "isa_merge_backward_tiles", "isa_set_tile_flow", "isa_tile_flow", "isa_ctx_set_params", "isa_batch_plan", "isa_ctx_set_tuning",
    "isa_batch_graph_create", "isa_batch_graph_launch", "isa_batch_graph_destroy", "isa_debayer_full", "isa_gamma_srgb",
    "isa_bw_image", "isa_prealign_burst", "isa_merge_backward", "isa_merge_batch", "isa_fourier_filter", "isa_gauss_filter", "isa_resize_box", "isa_track_level", "isa_upsample_shifts",
    "isa_solve_shifts", "isa_solve_shifts_static", "isa_optimal_shifts", "isa_flow_from_tiles", "isa_warp", "isa_derivatives", "isa_derivatives2",
    "isa_lucas_kanade", "isa_lk_iteration", "isa_lk_refine", "isa_debayer_subsample", "isa_robustness_mask", "isa_erode",
    "isa_robustness_erode", "isa_structure_tensor", "isa_kernel_param", "isa_accumulate", "isa_apply_weighting",
    "isa_color_twists", "isa_postprocess", "isa_save_tiff16", "isa_save_as_16bit_tiff",
    "isa_pef_huff_table", "isa_pef_decode_scratch", "isa_pef_decode", "isa_pef_unpack", "isa_pef_levels",
    "isa_dng_color_spec", "isa_pef_color_spec", "isa_dng_decode_scratch", "isa_dng_decode",
    "isa_dng_levels", "isa_noise_model", "isa_crop_window", "isa_profile_color_spec", "isa_dng_decode_path",
    "isa_dng_open", "isa_dng_close", "isa_dng_file_info", "isa_dng_roll_angle", "isa_dng_decode_begin", "isa_dng_decode_finish", "isa_pef_open", "isa_pef_close", "isa_pef_file_info",
]

_lib = None


def lib():
    """Load libisa.so (building it first if the sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        if not os.path.exists(LIB_PATH):
            raise IsaError(ISA_EINVAL, f"{LIB_PATH} is missing; build it with python -m imagestackalignator_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        L.isa_last_error.restype = ctypes.c_char_p
        L.isa_version.restype = ctypes.c_char_p
        for name in EXPORTS:
            f = getattr(L, name)
            if name not in ("isa_last_error", "isa_version", "isa_params_default"):
                f.restype = ctypes.c_int
        L.isa_launch_count.restype = ctypes.c_long
        L.isa_pef_decode_scratch.restype = ctypes.c_size_t
        L.isa_dng_decode_scratch.restype = ctypes.c_size_t
        _lib = L
    return _lib


def check(code):
    if code != ISA_OK:
        raise IsaError(code, lib().isa_last_error().decode())
    return code


def vp(x):
    """Device pointer of a torch tensor (or an int / None)."""
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    return ctypes.c_void_p(x.data_ptr())


def stream_ptr(stream=None):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def make_params(p: Optional[P.MergeParams] = None, fused_accumulate=True) -> IsaParams:
    p = p or P.MergeParams()
    c = IsaParams()
    lib().isa_params_default(ctypes.byref(c))
    for name in ("sigma_debayer_tracking", "sigma_debayer_accumulation", "high_pass", "high_pass_sigma", "matching_threshold",
                 "sigma_structure_tensor", "dth", "dtr", "k_detail", "k_denoise", "k_stretch", "k_shrink", "min_det_lk", "threshold_m",
                 "merge_scale", "robust_s", "robust_t"):
        setattr(c, name, float(getattr(p, name)))
    for name in ("clear_axis", "iterations_lk", "window_size_lk", "erode_size", "tracking_strategy", "tracking_block_size", "sample_mode"):
        setattr(c, name, int(getattr(p, name)))
    c.green_channel_only = int(bool(p.green_channel_only))
    c.super_resolution = int(bool(p.super_resolution))
    c.level_count = len(p.levels)
    for i, lv in enumerate(p.levels):
        c.levels[i] = IsaLevel(lv.resize_level, lv.tile_size, lv.max_shift)
    c.fused_accumulate = int(bool(fused_accumulate))
    return c


def make_info(burst) -> IsaRawInfo:
    i = IsaRawInfo()
    i.width, i.height = burst.width, burst.height
    for k in range(4):
        i.cfa[k] = int(burst.cfa[k])
    for k in range(3):
        i.black[k] = float(burst.black[k])
        i.white[k] = float(burst.white[k])
        i.camera_white[k] = float(burst.camera_white[k])
    i.noise_alpha = float(burst.noise_a)
    i.noise_beta = float(burst.noise_b)
    return i


def tracking_pairs(n, reference, strategy, block):
    """(pairs m x 2 in tracking order, rows m x 3 = (a, b, sign) per measurement row)."""
    m = lib().isa_tracking_pairs(n, reference, strategy, block, None, None, 0)
    check(m if m < 0 else 0)
    pairs = np.zeros((m, 2), np.int32)
    rows = np.zeros((m, 3), np.int32)
    got = lib().isa_tracking_pairs(n, reference, strategy, block, pairs.ctypes.data_as(ctypes.c_void_p),
                                   rows.ctypes.data_as(ctypes.c_void_p), m)
    check(got if got < 0 else 0)
    return pairs, rows


def output_size(p: IsaParams, width, height):
    w, h = ctypes.c_int(), ctypes.c_int()
    check(lib().isa_output_size(ctypes.byref(p), width, height, ctypes.byref(w), ctypes.byref(h)))
    return w.value, h.value


class Merger:
    """Owns an isa_ctx: the B200 counterpart of the controller's
    TrackPatches + PrepareAccumulation + Accumulate for one burst size."""

    def __init__(self, max_width, max_height, max_frames, params: Optional[P.MergeParams] = None, fused_accumulate=True):
        self.params = make_params(params, fused_accumulate)
        self.ctx = ctypes.c_void_p()
        check(lib().isa_ctx_create(ctypes.byref(self.ctx), max_width, max_height, max_frames, ctypes.byref(self.params)))

    def close(self):
        if self.ctx:
            lib().isa_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def output_size(self, width, height):
        return output_size(self.params, width, height)

    @staticmethod
    def _pre(n, shifts=None, rotations=None, reference=0):
        pre = IsaPrealign()
        keep = []
        if shifts is not None:
            a = np.ascontiguousarray(shifts, dtype=np.float32).reshape(n, 2)
            keep.append(a)
            pre.shifts = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        if rotations is not None:
            r = np.ascontiguousarray(rotations, dtype=np.float32).reshape(n)
            keep.append(r)
            pre.rotations_deg = r.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        pre.reference = int(reference)
        return pre, keep

    def merge(self, raw, info: IsaRawInfo, out=None, shifts=None, rotations=None, reference=0, stream=None):
        """raw: cuda uint16-compatible tensor n x H x W (torch.int16/uint16 storage); returns out (Ho x Wo x 3 float32)."""
        import torch
        n, H, W = raw.shape
        Wo, Ho = self.output_size(W, H)
        if out is None:
            out = torch.empty((Ho, Wo, 3), dtype=torch.float32, device=raw.device)
        pre, keep = self._pre(n, shifts, rotations, reference)
        check(lib().isa_merge_burst(self.ctx, vp(raw), ctypes.c_size_t(W * 2), ctypes.c_size_t(W * H * 2), n, ctypes.byref(info),
                                    ctypes.byref(pre), vp(out), ctypes.c_size_t(Wo * 12), stream_ptr(stream)))
        return out

    def backward(self, raw, info: IsaRawInfo, target, weight=None, out=None, shifts=None, rotations=None, reference=0, stream=None):
        """Forward merge and the adjoint of sum(weight * (out - target)^2) (isa_merge_backward).

        Returns (out, loss, grad) with grad = d loss / d (k_detail, k_denoise,
        dth, dtr, k_stretch, k_shrink, robust_s, robust_t) as float64."""
        import torch
        n, H, W = raw.shape
        Wo, Ho = self.output_size(W, H)
        if out is None:
            out = torch.empty((Ho, Wo, 3), dtype=torch.float32, device=raw.device)
        pre, keep = self._pre(n, shifts, rotations, reference)
        loss = ctypes.c_double()
        grad = np.zeros(8, np.float64)
        check(lib().isa_merge_backward(self.ctx, vp(raw), ctypes.c_size_t(W * 2), ctypes.c_size_t(W * H * 2), n, ctypes.byref(info),
                                       ctypes.byref(pre), vp(target), ctypes.c_size_t(Wo * 12), vp(weight) if weight is not None else None,
                                       ctypes.c_size_t(Wo * 4), vp(out), ctypes.c_size_t(Wo * 12),
                                       ctypes.byref(loss), grad.ctypes.data_as(ctypes.c_void_p), stream_ptr(stream)))
        return out, loss.value, grad

    def backward_tiles(self, raw, info: IsaRawInfo, target, weight=None, out=None, shifts=None, rotations=None, reference=0, stream=None):
        """isa_merge_backward_tiles: (out, loss, grad, tile_grad) with tile_grad
        = d loss / d (tile flow), a cuda float32 tensor n x tiles_y x tiles_x x 2
        (the context must use sample_mode SAMPLE_BILINEAR)."""
        import torch
        n, H, W = raw.shape
        Wo, Ho = self.output_size(W, H)
        if out is None:
            out = torch.empty((Ho, Wo, 3), dtype=torch.float32, device=raw.device)
        tx, ty = self.tile_grid(W, H)
        tg = torch.empty((n, ty, tx, 2), dtype=torch.float32, device=raw.device)
        pre, keep = self._pre(n, shifts, rotations, reference)
        loss = ctypes.c_double()
        grad = np.zeros(8, np.float64)
        check(lib().isa_merge_backward_tiles(self.ctx, vp(raw), ctypes.c_size_t(W * 2), ctypes.c_size_t(W * H * 2), n, ctypes.byref(info),
                                             ctypes.byref(pre), vp(target), ctypes.c_size_t(Wo * 12),
                                             vp(weight) if weight is not None else None, ctypes.c_size_t(Wo * 4), vp(out),
                                             ctypes.c_size_t(Wo * 12), ctypes.byref(loss), grad.ctypes.data_as(ctypes.c_void_p), vp(tg),
                                             stream_ptr(stream)))
        return out, loss.value, grad, tg

    def tile_grid(self, width, height):
        """Tile counts (tiles_x, tiles_y) of the finest tracking level for a width x height frame."""
        lv = self.params.levels[0]
        return ((width // lv.resize_level - 2 * lv.max_shift) // lv.tile_size, (height // lv.resize_level - 2 * lv.max_shift) // lv.tile_size)

    def set_params(self, params: P.MergeParams):
        """Replace the context's parameters (isa_ctx_set_params): same levels and tracking, output within the context."""
        c = make_params(params, bool(self.params.fused_accumulate))
        check(lib().isa_ctx_set_params(self.ctx, ctypes.byref(c)))
        self.params = c

    def set_tuning(self, entries=()):
        """isa_ctx_set_tuning: launch shapes per frame size, each entry a dict with width, height (0, 0: any size),
        lk_strip_rows, acc_block_x, acc_block_y (0: the library's choice)."""
        arr = (IsaTuning * max(1, len(entries)))()
        for i, e in enumerate(entries):
            arr[i] = IsaTuning(int(e.get("width", 0)), int(e.get("height", 0)), int(e.get("lk_strip_rows", 0)), int(e.get("acc_block_x", 0)),
                               int(e.get("acc_block_y", 0)))
        check(lib().isa_ctx_set_tuning(self.ctx, arr, len(entries)))

    def set_tile_flow(self, tiles=None):
        """Merge at the given per-frame tile flows (cuda float32 n x tiles_y x
        tiles_x x 2, kept alive by the caller) instead of the solved ones; None
        returns to the solved flows (isa_set_tile_flow)."""
        self._tile_override = tiles
        check(lib().isa_set_tile_flow(self.ctx, vp(tiles) if tiles is not None else None))

    def tile_flow(self, n, stream=None):
        """The last merge's per-frame tile flows (isa_tile_flow) as a cuda tensor n x tiles_y x tiles_x x 2."""
        import torch
        tx, ty = ctypes.c_int(), ctypes.c_int()
        check(lib().isa_tile_flow(self.ctx, None, ctypes.byref(tx), ctypes.byref(ty), stream_ptr(stream)))
        t = torch.empty((n, ty.value, tx.value, 2), dtype=torch.float32, device="cuda")
        check(lib().isa_tile_flow(self.ctx, vp(t), None, None, stream_ptr(stream)))
        return t

    def merge_host(self, raw_host, info: IsaRawInfo, out_host=None, shifts=None, rotations=None, reference=0, stream=None):
        """raw_host: host uint16 array/tensor (pinned for full speed); returns host float32 Ho x Wo x 3."""
        n, H, W = raw_host.shape
        Wo, Ho = self.output_size(W, H)
        if out_host is None:
            out_host = np.empty((Ho, Wo, 3), np.float32)
        pre, keep = self._pre(n, shifts, rotations, reference)
        rp = ctypes.c_void_p(raw_host.data_ptr()) if hasattr(raw_host, "data_ptr") else raw_host.ctypes.data_as(ctypes.c_void_p)
        op = ctypes.c_void_p(out_host.data_ptr()) if hasattr(out_host, "data_ptr") else out_host.ctypes.data_as(ctypes.c_void_p)
        check(lib().isa_merge_burst_host(self.ctx, rp, n, ctypes.byref(info), ctypes.byref(pre), op, stream_ptr(stream)))
        return out_host

    def prealign(self, raw, info: IsaRawInfo, increment=0.1, range_deg=1.0, roll=None, stream=None):
        """Global pre-alignment (isa_prealign_burst) of a device burst n x H x W.

        Returns (shifts n x 2, rotations_deg n, reference, scan n x 4): the
        PreAlignmentStore outputs that `merge(..., shifts=, rotations=,
        reference=)` takes, and the raw per-frame scan results against frame 0."""
        n, H, W = raw.shape
        shifts = np.zeros((n, 2), np.float32)
        rots = np.zeros(n, np.float32)
        scan = np.zeros((n, 4), np.float64)
        ref = ctypes.c_int(-1)
        rl = None
        if roll is not None:
            rl = np.ascontiguousarray(roll, dtype=np.float32)
        check(lib().isa_prealign_burst(self.ctx, vp(raw), ctypes.c_size_t(W * 2), ctypes.c_size_t(W * H * 2), n, ctypes.byref(info),
                                       ctypes.c_float(increment), ctypes.c_float(range_deg),
                                       rl.ctypes.data_as(ctypes.c_void_p) if rl is not None else None,
                                       shifts.ctypes.data_as(ctypes.c_void_p), rots.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ref),
                                       scan.ctypes.data_as(ctypes.c_void_p), stream_ptr(stream)))
        return shifts, rots, ref.value, scan

    def stage_times(self):
        ms = (ctypes.c_float * 8)()
        k = lib().isa_stage_times(self.ctx, ms, 8)
        if k < 0:
            check(k)
        return [ms[i] for i in range(k)]

    def launch_count(self):
        return int(lib().isa_launch_count(self.ctx))

    def debug(self, frame):
        ptrs = [ctypes.c_void_p() for _ in range(7)]
        pitches = [ctypes.c_size_t() for _ in range(4)]
        check(lib().isa_debug_buffers(self.ctx, frame, ctypes.byref(ptrs[0]), ctypes.byref(pitches[0]), ctypes.byref(ptrs[1]),
                                      ctypes.byref(pitches[1]), ctypes.byref(ptrs[2]), ctypes.byref(pitches[2]), ctypes.byref(ptrs[3]),
                                      ctypes.byref(ptrs[4]), ctypes.byref(pitches[3]), ctypes.byref(ptrs[5]), ctypes.byref(ptrs[6]),
                                      ctypes.byref(ctypes.c_size_t())))
        return {"flow": ptrs[0].value, "mask": ptrs[1].value, "kparam": ptrs[2].value, "bw_track": ptrs[3].value,
                "bw_acc": ptrs[4].value, "acc": ptrs[5].value, "wsum": ptrs[6].value}

    def debug_shifts(self):
        p = ctypes.c_void_p()
        tx, ty = ctypes.c_int(), ctypes.c_int()
        check(lib().isa_debug_shifts(self.ctx, ctypes.byref(p), ctypes.byref(tx), ctypes.byref(ty)))
        return p.value, tx.value, ty.value

    def set_track_record(self, record=None):
        """Record every level's integer tile shifts and search-block offsets of
        the following merges into `record` (a cuda int32 tensor; None stops)."""
        if record is None:
            check(lib().isa_debug_track_record(self.ctx, None, ctypes.c_size_t(0)))
        else:
            check(lib().isa_debug_track_record(self.ctx, vp(record), ctypes.c_size_t(record.numel() * record.element_size())))

    def flows_masks(self, n, width, height, reference=0):
        """Dense flows (H x W x 2) and eroded masks (H/2 x W/2 x 4) of the last
        merge, as host float32 arrays keyed by frame (the reference excluded)."""
        import torch
        flows, masks = {}, {}
        for i in range(n):
            if i == reference:
                continue
            d = self.debug(i)
            flows[i] = device_copy(d["flow"], (height, width, 2), torch.float32).cpu().numpy()
            masks[i] = device_copy(d["mask"], (height // 2, width // 2, 4), torch.float32).cpu().numpy()
        return flows, masks


    def kernel_params(self, width, height):
        """Kernel parameters of the last merge's reference frame (H x W x 4, host float32)."""
        import torch
        return device_copy(self.debug(0)["kparam"], (height, width, 4), torch.float32).cpu().numpy()

    def weight_sums(self, width, height):
        """Per-channel weight sums of the last merge's accumulation (Ho x Wo x 3, host float32)."""
        import torch
        Wo, Ho = self.output_size(width, height)
        return device_copy(self.debug(0)["wsum"], (Ho, Wo, 3), torch.float32).cpu().numpy()


def track_record_ints(params: IsaParams, width, height, npairs):
    """int32 entries of an isa_debug_track_record buffer for one merge."""
    total = 0
    for li in range(params.level_count):
        lv = params.levels[li]
        tcx = (width // lv.resize_level - 2 * lv.max_shift) // lv.tile_size
        tcy = (height // lv.resize_level - 2 * lv.max_shift) // lv.tile_size
        total += 3 * npairs * tcx * tcy
    return total


MAX_LUT = 512
POST_RGB16, POST_BGRA8 = 0, 1


class IsaPostParams(ctypes.Structure):
    _fields_ = [("crop_x", ctypes.c_int), ("crop_y", ctypes.c_int), ("crop_w", ctypes.c_int), ("crop_h", ctypes.c_int),
                ("camera_white", ctypes.c_float * 3), ("twist1", ctypes.c_float * 12), ("twist2", ctypes.c_float * 12),
                ("lut_x", ctypes.c_void_p), ("lut_y", ctypes.c_void_p), ("nlut", ctypes.c_int), ("exposure", ctypes.c_float)]


def color_twists(camera_to_pcs):
    """isa_color_twists: (camera -> ProPhoto, ProPhoto -> sRGB) as float32 3 x 4 arrays."""
    m = np.ascontiguousarray(camera_to_pcs, np.float64).reshape(9)
    t1 = np.zeros(12, np.float32)
    t2 = np.zeros(12, np.float32)
    check(lib().isa_color_twists(m.ctypes.data_as(ctypes.c_void_p), t1.ctypes.data_as(ctypes.c_void_p), t2.ctypes.data_as(ctypes.c_void_p)))
    return t1.reshape(3, 4), t2.reshape(3, 4)


def post_params(crop, camera_white, twist1, twist2, lut_x, lut_y, exposure=0.0):
    """(IsaPostParams, arrays to keep alive while it is used)."""
    lx = np.ascontiguousarray(lut_x, np.float32)
    ly = np.ascontiguousarray(lut_y, np.float32)
    pp = IsaPostParams()
    pp.crop_x, pp.crop_y, pp.crop_w, pp.crop_h = (int(v) for v in crop)
    for c in range(3):
        pp.camera_white[c] = float(camera_white[c])
    for i, v in enumerate(np.asarray(twist1, np.float32).reshape(12)):
        pp.twist1[i] = float(v)
    for i, v in enumerate(np.asarray(twist2, np.float32).reshape(12)):
        pp.twist2[i] = float(v)
    pp.lut_x = lx.ctypes.data
    pp.lut_y = ly.ctypes.data
    pp.nlut = len(lx)
    pp.exposure = float(exposure)
    return pp, (lx, ly)


def postprocess(img, pp: IsaPostParams, fmt=POST_RGB16, out=None, stream=None):
    """isa_postprocess on a device float32 H x W x 3 image; returns the crop as
    uint16 crop_h x crop_w x 3 (RGB16) or uint8 crop_h x crop_w x 4 (BGRA8)."""
    import torch
    H, W, _ = img.shape
    if out is None:
        shape = (pp.crop_h, pp.crop_w, 3) if fmt == POST_RGB16 else (pp.crop_h, pp.crop_w, 4)
        out = torch.empty(shape, dtype=torch.int16 if fmt == POST_RGB16 else torch.uint8, device=img.device)
    row = pp.crop_w * (6 if fmt == POST_RGB16 else 4)
    check(lib().isa_postprocess(vp(img), ctypes.c_size_t(W * 12), W, H, ctypes.byref(pp), fmt, vp(out), ctypes.c_size_t(row),
                                stream_ptr(stream)))
    return out


def save_tiff16(path, rgb):
    """isa_save_tiff16 of a host uint16 H x W x 3 array."""
    a = np.ascontiguousarray(rgb, np.uint16)
    h, w, _ = a.shape
    check(lib().isa_save_tiff16(os.fsencode(path), a.ctypes.data_as(ctypes.c_void_p), w, h))


def save_as_16bit_tiff(img, pp: IsaPostParams, path, stream=None):
    """isa_save_as_16bit_tiff: post-process a device float3 image and write the TIFF."""
    H, W, _ = img.shape
    check(lib().isa_save_as_16bit_tiff(vp(img), ctypes.c_size_t(W * 12), W, H, ctypes.byref(pp), os.fsencode(path), stream_ptr(stream)))


def pef_huff_table(maker_note: bytes, big_endian=False):
    """isa_pef_huff_table: the 4097-entry decode table from the HuffmanTable maker-note bytes."""
    buf = np.frombuffer(bytes(maker_note), np.uint8).copy()
    t = np.zeros(4097, np.uint16)
    n = lib().isa_pef_huff_table(buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(buf.size), int(big_endian), t.ctypes.data_as(ctypes.c_void_p))
    check(n if n < 0 else 0)
    return t


def pef_decode(data, table, width, height, out=None, scratch=None, stream=None):
    """isa_pef_decode of a device uint8 stream; returns the uint16 height x
    width frame as an int16 tensor."""
    import torch
    nbytes = data.numel()
    need = lib().isa_pef_decode_scratch(ctypes.c_size_t(nbytes), width, height)
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(need, dtype=torch.uint8, device=data.device)
    if out is None:
        out = torch.empty((height, width), dtype=torch.int16, device=data.device)
    t = np.ascontiguousarray(table, np.uint16)
    check(lib().isa_pef_decode(vp(data), ctypes.c_size_t(nbytes), t.ctypes.data_as(ctypes.c_void_p), width, height, vp(scratch),
                               ctypes.c_size_t(scratch.numel()), vp(out), ctypes.c_size_t(out.stride(0) * 2), stream_ptr(stream)))
    return out


def pef_unpack(file, offsets, sizes, rows_per_strip, width, height, bit_depth, out=None, stream=None):
    """isa_pef_unpack of a device uint8 file image; returns the frame (int16 tensor holding uint16)."""
    import torch
    off = np.ascontiguousarray(offsets, np.uint32)
    sz = np.ascontiguousarray(sizes, np.uint32)
    if out is None:
        out = torch.empty((height, width), dtype=torch.int16, device=file.device)
    check(lib().isa_pef_unpack(vp(file), ctypes.c_size_t(file.numel()), off.ctypes.data_as(ctypes.c_void_p), sz.ctypes.data_as(ctypes.c_void_p),
                               len(off), rows_per_strip, width, height, bit_depth, vp(out), ctypes.c_size_t(out.stride(0) * 2),
                               stream_ptr(stream)))
    return out


def pef_levels(cfa, black_point, white_level, white_point, scaling, bit_depth):
    """isa_pef_levels: (black[3], white[3], white_balance[3]) as float32 arrays."""
    c = np.ascontiguousarray(cfa, np.int32)
    bp = np.ascontiguousarray([] if black_point is None else black_point, np.float32)
    wp = np.ascontiguousarray(white_point, np.float32)
    b = np.zeros(3, np.float32)
    w = np.zeros(3, np.float32)
    wb = np.zeros(3, np.float32)
    check(lib().isa_pef_levels(c.ctypes.data_as(ctypes.c_void_p), bp.ctypes.data_as(ctypes.c_void_p) if bp.size else None, int(bp.size),
                               ctypes.c_float(-1.0 if white_level is None else float(white_level)), wp.ctypes.data_as(ctypes.c_void_p),
                               ctypes.c_float(scaling), bit_depth, b.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p),
                               wb.ctypes.data_as(ctypes.c_void_p)))
    return b, w, wb


class IsaDngColorTags(ctypes.Structure):
    _fields_ = [("color_matrix1", ctypes.c_void_p), ("color_matrix2", ctypes.c_void_p), ("illuminant1", ctypes.c_int),
                ("illuminant2", ctypes.c_int), ("forward_matrix1", ctypes.c_void_p), ("forward_matrix2", ctypes.c_void_p),
                ("camera_calibration1", ctypes.c_void_p), ("camera_calibration2", ctypes.c_void_p), ("analog_balance", ctypes.c_void_p),
                ("as_shot_neutral", ctypes.c_void_p), ("as_shot_white_xy", ctypes.c_void_p)]


def dng_color_spec(color_matrix1=None, color_matrix2=None, illuminant1=0, illuminant2=0, forward_matrix1=None, forward_matrix2=None,
                   camera_calibration1=None, camera_calibration2=None, analog_balance=None, as_shot_neutral=None, as_shot_white_xy=None):
    """isa_dng_color_spec: (camera_to_pcs 3 x 3, camera_white 3, white xy 2) as float64."""
    keep = []

    def arr(v, n):
        if v is None:
            return None
        a = np.ascontiguousarray(v, np.float64).reshape(n)
        keep.append(a)
        return a.ctypes.data

    t = IsaDngColorTags(arr(color_matrix1, 9), arr(color_matrix2, 9), int(illuminant1), int(illuminant2), arr(forward_matrix1, 9),
                        arr(forward_matrix2, 9), arr(camera_calibration1, 9), arr(camera_calibration2, 9), arr(analog_balance, 3),
                        arr(as_shot_neutral, 3), arr(as_shot_white_xy, 2))
    c2p = np.zeros(9)
    cw = np.zeros(3)
    xy = np.zeros(2)
    check(lib().isa_dng_color_spec(ctypes.byref(t), c2p.ctypes.data_as(ctypes.c_void_p), cw.ctypes.data_as(ctypes.c_void_p),
                                   xy.ctypes.data_as(ctypes.c_void_p)))
    return c2p.reshape(3, 3), cw, xy


def pef_color_spec(white_balance):
    """isa_pef_color_spec: the colour spec of a PEF file from its white balance."""
    wb = np.ascontiguousarray(white_balance, np.float32)
    c2p = np.zeros(9)
    cw = np.zeros(3)
    xy = np.zeros(2)
    check(lib().isa_pef_color_spec(wb.ctypes.data_as(ctypes.c_void_p), c2p.ctypes.data_as(ctypes.c_void_p), cw.ctypes.data_as(ctypes.c_void_p),
                                   xy.ctypes.data_as(ctypes.c_void_p)))
    return c2p.reshape(3, 3), cw, xy


def profile_color_spec(white_balance, color_matrix1=None, color_matrix2=None, illuminant1=0, illuminant2=0):
    """isa_profile_color_spec: the colour spec of a camera profile (matrices, illuminants) and a white balance."""
    keep = []

    def arr(v):
        if v is None:
            return None
        a = np.ascontiguousarray(v, np.float64).reshape(9)
        keep.append(a)
        return a.ctypes.data_as(ctypes.c_void_p)

    wb = np.ascontiguousarray(white_balance, np.float32)
    c2p = np.zeros(9)
    cw = np.zeros(3)
    xy = np.zeros(2)
    check(lib().isa_profile_color_spec(arr(color_matrix1), arr(color_matrix2), int(illuminant1), int(illuminant2),
                                       wb.ctypes.data_as(ctypes.c_void_p), c2p.ctypes.data_as(ctypes.c_void_p),
                                       cw.ctypes.data_as(ctypes.c_void_p), xy.ctypes.data_as(ctypes.c_void_p)))
    return c2p.reshape(3, 3), cw, xy


def noise_model(iso, isos, alpha, beta):
    """isa_noise_model: (alpha, beta) of a camera profile's noise model at `iso`."""
    i = np.ascontiguousarray(isos, np.int32)
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(beta, np.float64)
    ab = np.zeros(2)
    check(lib().isa_noise_model(int(iso), i.ctypes.data_as(ctypes.c_void_p), a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                                int(i.size), ab.ctypes.data_as(ctypes.c_void_p)))
    return float(ab[0]), float(ab[1])


def crop_window(left, top, cropped_width, cropped_height, width, height):
    """isa_crop_window: (left, top, width, height) kept at least two pixels off the frame's edges."""
    c = (ctypes.c_int * 4)()
    check(lib().isa_crop_window(int(left), int(top), int(cropped_width), int(cropped_height), int(width), int(height), c))
    return tuple(c)


class IsaDngLevelTags(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("cfa_pattern", ctypes.c_void_p), ("cfa_repeat_w", ctypes.c_int),
                ("cfa_repeat_h", ctypes.c_int), ("plane_color", ctypes.c_void_p), ("n_plane_color", ctypes.c_int),
                ("black_level", ctypes.c_void_p), ("n_black", ctypes.c_int), ("white_level", ctypes.c_double),
                ("camera_white", ctypes.c_void_p), ("active_area", ctypes.c_void_p), ("default_crop_origin", ctypes.c_void_p),
                ("default_crop_size", ctypes.c_void_p), ("noise_profile", ctypes.c_void_p), ("n_noise", ctypes.c_int),
                ("black_delta_h", ctypes.c_void_p), ("n_delta_h", ctypes.c_int), ("black_delta_v", ctypes.c_void_p),
                ("n_delta_v", ctypes.c_int), ("iso", ctypes.c_int), ("profile_iso", ctypes.c_void_p), ("profile_alpha", ctypes.c_void_p),
                ("profile_beta", ctypes.c_void_p), ("n_profile", ctypes.c_int)]


class IsaRawLevels(ctypes.Structure):
    _fields_ = [("info", IsaRawInfo), ("white_balance", ctypes.c_float * 3), ("color_twist", ctypes.c_float * 12),
                ("color_twist_identity", ctypes.c_int), ("crop", ctypes.c_int * 4)]


def dng_levels(width, height, cfa_pattern, white_level, camera_white, cfa_repeat=(2, 2), plane_color=None, black_level=None,
               active_area=None, default_crop_origin=None, default_crop_size=None, noise_profile=None, black_delta_h=None,
               black_delta_v=None, iso=0, profile_noise=None):
    """isa_dng_levels. profile_noise = (isos, alphas, betas) of an ExtraCameraProfiles entry, or None.
    Returns a dict of the levels plus the placed black deltas (uint16 width and height entries)."""
    keep = []

    def arr(v, dt):
        if v is None:
            return None, 0
        a = np.ascontiguousarray(v, dt).reshape(-1)
        keep.append(a)
        return a.ctypes.data, int(a.size)

    cfa, _ = arr(cfa_pattern, np.uint8)
    pc, npc = arr(plane_color, np.int32)
    bl, nbl = arr(black_level, np.float64)
    cw, _ = arr(camera_white, np.float64)
    aa, _ = arr(active_area, np.int32)
    co, _ = arr(default_crop_origin, np.float64)
    cs, _ = arr(default_crop_size, np.float64)
    npf, nn = arr(noise_profile, np.float64)
    dh, ndh = arr(black_delta_h, np.float64)
    dv, ndv = arr(black_delta_v, np.float64)
    pi, npi = arr(None if profile_noise is None else profile_noise[0], np.int32)
    pa, _ = arr(None if profile_noise is None else profile_noise[1], np.float64)
    pb, _ = arr(None if profile_noise is None else profile_noise[2], np.float64)
    t = IsaDngLevelTags(width, height, cfa, cfa_repeat[0], cfa_repeat[1], pc, npc, bl, nbl, float(white_level), cw, aa, co, cs, npf, nn, dh, ndh,
                        dv, ndv, int(iso), pi, pa, pb, npi)
    r = IsaRawLevels()
    bh = np.zeros(width, np.uint16)
    bv = np.zeros(height, np.uint16)
    check(lib().isa_dng_levels(ctypes.byref(t), ctypes.byref(r), bh.ctypes.data_as(ctypes.c_void_p), bv.ctypes.data_as(ctypes.c_void_p)))
    i = r.info
    return dict(cfa=list(i.cfa), black=np.array(i.black, np.float32), white=np.array(i.white, np.float32),
                camera_white=np.array(i.camera_white, np.float32), noise=(np.float32(i.noise_alpha), np.float32(i.noise_beta)),
                white_balance=np.array(r.white_balance, np.float32), color_twist=np.array(r.color_twist, np.float32).reshape(3, 4),
                color_twist_identity=bool(r.color_twist_identity), crop=tuple(r.crop), black_h=bh, black_v=bv, info=i)


def dng_decode_path():
    """isa_dng_decode_path: 1 parallel decoder, 0 per-part reader, -1 none (the calling thread's last isa_dng_decode)."""
    return int(lib().isa_dng_decode_path())


class IsaDngLayout(ctypes.Structure):
    _fields_ = [("tiled", ctypes.c_int), ("tile_width", ctypes.c_int), ("tile_height", ctypes.c_int), ("rows_per_strip", ctypes.c_int),
                ("n", ctypes.c_int), ("offsets", ctypes.c_void_p), ("byte_counts", ctypes.c_void_p), ("compression", ctypes.c_int),
                ("bit_depth", ctypes.c_int), ("dng_version_large", ctypes.c_int), ("linearization", ctypes.c_void_p), ("nlin", ctypes.c_int),
                ("black_h", ctypes.c_void_p), ("black_v", ctypes.c_void_p)]


def dng_decode(file, width, height, offsets, counts, compression=7, tiled=True, tile_w=0, tile_h=0, rows_per_strip=0, bit_depth=16, large=True,
               linearization=None, black_h=None, black_v=None, file_dev=None, stream=None, scratch=None, out=None, phase=None):
    """isa_dng_decode of a DNG file image (host uint8 array; copied to the
    device unless file_dev is given); returns the frame (int16 tensor holding
    uint16). scratch / out: device buffers to reuse (scratch of at least
    isa_dng_decode_scratch bytes). phase "begin" / "finish": the two halves
    (isa_dng_decode_begin / _finish), called with the same arguments."""
    import torch
    f = np.ascontiguousarray(file, np.uint8)
    keep = [np.ascontiguousarray(offsets, np.uint32), np.ascontiguousarray(counts, np.uint32)]
    lin = None if linearization is None else np.ascontiguousarray(linearization, np.uint16)
    bh = None if black_h is None else np.ascontiguousarray(black_h, np.uint16)
    bv = None if black_v is None else np.ascontiguousarray(black_v, np.uint16)
    keep += [lin, bh, bv]
    L = IsaDngLayout(int(tiled), tile_w, tile_h, rows_per_strip, len(keep[0]), keep[0].ctypes.data, keep[1].ctypes.data, compression, bit_depth,
                     int(large), None if lin is None else lin.ctypes.data, 0 if lin is None else lin.size,
                     None if bh is None else bh.ctypes.data, None if bv is None else bv.ctypes.data)
    fp = f.ctypes.data_as(ctypes.c_void_p)
    dev = file_dev if file_dev is not None else torch.from_numpy(f).cuda()
    if scratch is None:
        need = lib().isa_dng_decode_scratch(fp, ctypes.c_size_t(f.size), ctypes.byref(L), width, height)
        if need == 0:
            raise IsaError(ISA_EINVAL, lib().isa_last_error().decode())
        scratch = torch.empty(need, dtype=torch.uint8, device=dev.device)
    if out is None:
        out = torch.empty((height, width), dtype=torch.int16, device=dev.device)
    fn = {None: lib().isa_dng_decode, "begin": lib().isa_dng_decode_begin, "finish": lib().isa_dng_decode_finish}[phase]
    check(fn(fp, vp(dev), ctypes.c_size_t(f.size), ctypes.byref(L), width, height, vp(scratch), ctypes.c_size_t(scratch.numel()),
             vp(out), ctypes.c_size_t(out.stride(0) * 2), stream_ptr(stream)))
    return out


def dng_decode_scratch(file, width, height, offsets, counts, compression=7, tiled=True, tile_w=0, tile_h=0, rows_per_strip=0, bit_depth=16,
                       large=True, linearization=None):
    """isa_dng_decode_scratch: device bytes isa_dng_decode needs for this file and layout."""
    f = np.ascontiguousarray(file, np.uint8)
    off = np.ascontiguousarray(offsets, np.uint32)
    cnt = np.ascontiguousarray(counts, np.uint32)
    nlin = 0 if linearization is None else len(linearization)
    L = IsaDngLayout(int(tiled), tile_w, tile_h, rows_per_strip, len(off), off.ctypes.data, cnt.ctypes.data, compression, bit_depth, int(large),
                     None, nlin, None, None)
    need = lib().isa_dng_decode_scratch(f.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(f.size), ctypes.byref(L), width, height)
    if need == 0:
        raise IsaError(ISA_EINVAL, lib().isa_last_error().decode())
    return int(need)


def _arr(ptr, n, ctype):
    if not ptr or n <= 0:
        return None
    return list(ctypes.cast(ptr, ctypes.POINTER(ctype))[:n])


def dng_open(file):
    """isa_dng_open + isa_dng_file_info of a DNG file image (host bytes): a dict
    with width, height and the keyword arguments of dng_decode ("layout"),
    dng_levels ("levels", without camera_white) and dng_color_spec ("color")."""
    f = np.ascontiguousarray(np.frombuffer(bytes(file), np.uint8) if isinstance(file, (bytes, bytearray)) else file, np.uint8)
    h = ctypes.c_void_p()
    check(lib().isa_dng_open(f.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(f.size), ctypes.byref(h)))
    try:
        L, G, C = IsaDngLayout(), IsaDngLevelTags(), IsaDngColorTags()
        W, H = ctypes.c_int(), ctypes.c_int()
        check(lib().isa_dng_file_info(h, ctypes.byref(L), ctypes.byref(G), ctypes.byref(C), ctypes.byref(W), ctypes.byref(H)))
        layout = dict(tiled=bool(L.tiled), tile_w=L.tile_width, tile_h=L.tile_height, rows_per_strip=L.rows_per_strip,
                      offsets=_arr(L.offsets, L.n, ctypes.c_uint32), counts=_arr(L.byte_counts, L.n, ctypes.c_uint32),
                      compression=L.compression, bit_depth=L.bit_depth, large=bool(L.dng_version_large),
                      linearization=_arr(L.linearization, L.nlin, ctypes.c_uint16))
        levels = dict(width=G.width, height=G.height, cfa_pattern=_arr(G.cfa_pattern, 4, ctypes.c_uint8),
                      cfa_repeat=(G.cfa_repeat_w, G.cfa_repeat_h), white_level=G.white_level,
                      plane_color=_arr(G.plane_color, G.n_plane_color, ctypes.c_int), black_level=_arr(G.black_level, G.n_black, ctypes.c_double),
                      active_area=_arr(G.active_area, 4, ctypes.c_int), default_crop_origin=_arr(G.default_crop_origin, 2, ctypes.c_double),
                      default_crop_size=_arr(G.default_crop_size, 2, ctypes.c_double),
                      noise_profile=_arr(G.noise_profile, G.n_noise, ctypes.c_double),
                      black_delta_h=_arr(G.black_delta_h, G.n_delta_h, ctypes.c_double),
                      black_delta_v=_arr(G.black_delta_v, G.n_delta_v, ctypes.c_double), iso=G.iso)
        color = dict(color_matrix1=_arr(C.color_matrix1, 9, ctypes.c_double), color_matrix2=_arr(C.color_matrix2, 9, ctypes.c_double),
                     illuminant1=C.illuminant1, illuminant2=C.illuminant2, forward_matrix1=_arr(C.forward_matrix1, 9, ctypes.c_double),
                     forward_matrix2=_arr(C.forward_matrix2, 9, ctypes.c_double),
                     camera_calibration1=_arr(C.camera_calibration1, 9, ctypes.c_double),
                     camera_calibration2=_arr(C.camera_calibration2, 9, ctypes.c_double),
                     analog_balance=_arr(C.analog_balance, 3, ctypes.c_double), as_shot_neutral=_arr(C.as_shot_neutral, 3, ctypes.c_double),
                     as_shot_white_xy=_arr(C.as_shot_white_xy, 2, ctypes.c_double))
        roll = ctypes.c_float()
        has_roll = lib().isa_dng_roll_angle(h, ctypes.byref(roll))
        return dict(width=W.value, height=H.value, layout=layout, levels=levels, color=color, roll_angle=float(roll.value) if has_roll == 1 else None)
    finally:
        lib().isa_dng_close(h)


class IsaPefInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("bit_depth", ctypes.c_int), ("cfa", ctypes.c_int * 4),
                ("nstrips", ctypes.c_int), ("rows_per_strip", ctypes.c_int), ("strip_offsets", ctypes.c_void_p),
                ("strip_sizes", ctypes.c_void_p), ("compressed", ctypes.c_int), ("huffman_table", ctypes.c_void_p),
                ("huffman_bytes", ctypes.c_size_t), ("huffman_big_endian", ctypes.c_int), ("black_point", ctypes.c_void_p),
                ("n_black", ctypes.c_int), ("white_level", ctypes.c_float), ("white_point", ctypes.c_float * 4), ("scaling", ctypes.c_float),
                ("iso", ctypes.c_int), ("roll_angle", ctypes.c_float), ("roll_angle_present", ctypes.c_int)]


def pef_open(file):
    """isa_pef_open + isa_pef_file_info of a PEF file image (host bytes) as a dict."""
    f = np.ascontiguousarray(np.frombuffer(bytes(file), np.uint8) if isinstance(file, (bytes, bytearray)) else file, np.uint8)
    h = ctypes.c_void_p()
    check(lib().isa_pef_open(f.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(f.size), ctypes.byref(h)))
    try:
        I = IsaPefInfo()
        check(lib().isa_pef_file_info(h, ctypes.byref(I)))
        huff = None
        if I.huffman_table:
            huff = bytes(ctypes.cast(I.huffman_table, ctypes.POINTER(ctypes.c_uint8))[:I.huffman_bytes])
        return dict(width=I.width, height=I.height, bit_depth=I.bit_depth, cfa=list(I.cfa), nstrips=I.nstrips, rows_per_strip=I.rows_per_strip,
                    strip_offsets=_arr(I.strip_offsets, I.nstrips, ctypes.c_uint32), strip_sizes=_arr(I.strip_sizes, I.nstrips, ctypes.c_uint32),
                    compressed=bool(I.compressed), huffman_table=huff, huffman_big_endian=bool(I.huffman_big_endian),
                    black_point=_arr(I.black_point, I.n_black, ctypes.c_float), white_level=None if I.white_level < 0 else I.white_level,
                    white_point=list(I.white_point), scaling=I.scaling, iso=I.iso,
                    roll_angle=float(I.roll_angle) if I.roll_angle_present else None)
    finally:
        lib().isa_pef_close(h)


class IsaBurst(ctypes.Structure):
    _fields_ = [("raw", ctypes.c_void_p), ("raw_pitch", ctypes.c_size_t), ("frame_stride", ctypes.c_size_t), ("n", ctypes.c_int),
                ("info", ctypes.c_void_p), ("pre", ctypes.c_void_p), ("params", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("out_pitch", ctypes.c_size_t)]


def merge_batch(mergers, bursts, streams=None):
    """isa_merge_batch: `bursts` is a list of dicts with raw (device n x H x W
    tensor), info (IsaRawInfo), out (device Ho x Wo x 3 tensor) and optionally
    params (MergeParams); returns the per-burst status list. Work is enqueued
    on `streams` (one per merger; torch streams or None) and not waited for."""
    keep = []
    arr = (IsaBurst * len(bursts))()
    for i, b in enumerate(bursts):
        raw, info, out = b["raw"], b["info"], b["out"]
        n, H, W = raw.shape
        pp = None
        if b.get("params") is not None:
            pp = make_params(b["params"])
            keep.append(pp)
        keep.append(info)
        arr[i] = IsaBurst(raw.data_ptr(), W * 2, W * H * 2, n, ctypes.addressof(info), None,
                          ctypes.addressof(pp) if pp is not None else None, out.data_ptr(), out.shape[1] * 12)
    ctxs = (ctypes.c_void_p * len(mergers))(*[m.ctx for m in mergers])
    sts = (ctypes.c_void_p * len(mergers))(*[stream_ptr(s) for s in (streams or [None] * len(mergers))])
    status = (ctypes.c_int * max(1, len(bursts)))()
    lib().isa_merge_batch(ctxs, sts, len(mergers), arr, len(bursts), status)
    return [status[i] for i in range(len(bursts))]


def _burst_array(bursts, keep):
    arr = (IsaBurst * len(bursts))()
    for i, b in enumerate(bursts):
        raw, info, out = b["raw"], b["info"], b["out"]
        n, H, W = raw.shape
        pp = None
        if b.get("params") is not None:
            pp = make_params(b["params"])
            keep.append(pp)
        keep.append(info)
        arr[i] = IsaBurst(raw.data_ptr(), W * 2, W * H * 2, n, ctypes.addressof(info), None,
                          ctypes.addressof(pp) if pp is not None else None, out.data_ptr(), out.shape[1] * 12)
    return arr


class BatchGraph:
    """A batch captured once as a CUDA graph (isa_batch_graph_create) and
    replayed with one host launch (isa_batch_graph_launch). `bursts` as for
    merge_batch; `streams`: one non-default torch stream per merger; the
    capture forks from and joins back to `origin` (a torch stream)."""

    def __init__(self, mergers, bursts, streams, origin):
        self._keep = []
        arr = _burst_array(bursts, self._keep)
        ctxs = (ctypes.c_void_p * len(mergers))(*[m.ctx for m in mergers])
        sts = (ctypes.c_void_p * len(mergers))(*[stream_ptr(s) for s in streams])
        self.g = ctypes.c_void_p()
        check(lib().isa_batch_graph_create(ctxs, sts, len(mergers), arr, len(bursts), stream_ptr(origin), ctypes.byref(self.g)))
        self._refs = (mergers, bursts, streams)

    def launch(self, stream=None):
        check(lib().isa_batch_graph_launch(self.g, stream_ptr(stream)))

    def close(self):
        if self.g:
            lib().isa_batch_graph_destroy(self.g)
            self.g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_plan(work, burst_device, ctx_device):
    """isa_batch_plan: the context index isa_merge_batch gives each burst (the
    least-loaded context, by W*H*n work in burst order, among those on the
    burst's device; -1 in burst_device = any device), -1 where none fits.
    Host only."""
    n, k = len(work), len(ctx_device)
    w = (ctypes.c_double * max(n, 1))(*[float(v) for v in work])
    bd = (ctypes.c_int * max(n, 1))(*[int(v) for v in burst_device])
    cd = (ctypes.c_int * k)(*[int(v) for v in ctx_device])
    out = (ctypes.c_int * max(n, 1))()
    r = lib().isa_batch_plan(w, bd, n, cd, k, out)
    if r < 0:
        check(r)
    return [out[i] for i in range(n)]


def rank_bursts(work, world):
    """Bursts of a batch shared out over `world` ranks (one process per GPU,
    each merging its own bursts, no collective on the data path): the same
    rule as isa_batch_plan with one context per rank, so every rank computes
    the same split from the same list. Returns, per rank, its burst indices."""
    plan = batch_plan(work, [-1] * len(work), list(range(world)))
    return [[b for b, r in enumerate(plan) if r == k] for k in range(world)]


def device_copy(ptr, shape, dtype, device="cuda"):
    """Copy `shape` elements of `dtype` from a device pointer into a new torch tensor."""
    import torch
    t = torch.empty(shape, dtype=dtype, device=device)
    s = torch.cuda.current_stream()
    rc = _cudart().cudaMemcpyAsync(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(ptr), ctypes.c_size_t(t.numel() * t.element_size()), 3,
                                   ctypes.c_void_p(s.cuda_stream))
    if rc != 0:
        raise IsaError(ISA_ECUDA, f"cudaMemcpyAsync failed ({rc})")
    return t


_CUDART = None


def _cudart():
    global _CUDART
    if _CUDART is None:
        import glob
        import torch
        cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib", "libcudart.so*"))
        cands += ["/usr/local/cuda/lib64/libcudart.so"]
        for c in cands:
            try:
                _CUDART = ctypes.CDLL(c)
                break
            except OSError:
                continue
        if _CUDART is None:
            raise IsaError(ISA_ECUDA, "libcudart not found")
    return _CUDART
