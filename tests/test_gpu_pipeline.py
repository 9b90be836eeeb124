"""Whole-burst merge on the GPU (isa_merge_burst) against the FP64 oracle, and
size-independent properties at the full 6016 x 4000 x 20 workload.

Tolerance of the merged image: max |GPU - FP64| <= 1e-4 of the white level
over every pixel whose discrete decisions match the oracle's. The merge
reads the flows only through round(s * flow) (DeBayerKernels.cu:310-311,
403-404) and round(flow / 2) (RobustnessModell.cu:401-402, through the
eroded mask), and ApplyWeighting tests w < threshold (kernel.cu:336-391); a
value within FP32 noise of a half-integer, or a flow that LK moved across
one in a nearly rank-one window next to the 2-px black demosaic border, can
decide the other way and change the pixel by up to the local contrast.
oracle/parity.py identifies those pixels from both sides' flows, masks and
weight sums, requires every differing mask value to be explained by a
differing rounding decision, and bounds their count. The oracle's
accumulation fed the GPU's own flows, masks and kernel parameters must
match the GPU to 1e-4 on every pixel; where only it matches (the kernel's
orientation is ill-conditioned where the structure tensor is nearly
isotropic, and at scales other than 1 and 2 a channel may be reached only by
far taps whose weights follow it), the pixel is counted as carried in from
upstream FP32 inputs."""
import ctypes

import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

import parity
import pipeline as PL

pytestmark = pytest.mark.gpu


def to_dev(raw):
    import torch
    return torch.from_numpy(np.ascontiguousarray(raw).view(np.int16)).cuda()


def gpu_merge(burst, p, fused=True, pre=None):
    import torch
    m = isa.Merger(burst.width, burst.height, burst.n, p, fused_accumulate=fused)
    info = isa.make_info(burst)
    kw = {}
    if pre is not None:
        kw = dict(shifts=pre.shifts, rotations=pre.rotations, reference=pre.reference)
    out = m.merge(to_dev(burst.raw), info, **kw)
    torch.cuda.synchronize()
    return m, out.cpu().numpy()


def image_parity(m, burst, p, got, want, keep, reference=0):
    """max |GPU - FP64| <= 1e-4 over the decision-matched pixels (oracle/parity.py)."""
    flows, masks = m.flows_masks(burst.n, burst.width, burst.height, reference=reference)
    geom = PL.out_geometry(burst.width, burst.height, p)
    sub = PL.merge_tail(burst, p, flows, masks, m.kernel_params(burst.width, burst.height), PL.StageLib("oracle64"), reference=reference)
    st = parity.merge_parity(got, want.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=want.wsum,
                             wsum_gpu=m.weight_sums(burst.width, burst.height), want_sub=sub.image, wsum_sub=sub.wsum, ref=reference)
    print(st)
    return st


@pytest.fixture(scope="module")
def burst():
    return synthetic.make_burst(640, 480, 5, seed=21, max_shift=6, max_rot_deg=0.2)


@pytest.mark.parametrize("mode", ["plain", "super", "x2", "x1.5"])
def test_merge_matches_oracle(cuda, oracle, burst, mode):
    p = P.MergeParams()
    p.super_resolution = mode == "super"
    p.merge_scale = {"x2": 2.0, "x1.5": 1.5}.get(mode, 0.0)
    keep = {}
    want = PL.merge_burst(burst, p, lib=oracle, keep=keep)
    m, got = gpu_merge(burst, p)
    image_parity(m, burst, p, got, want, keep)
    # intermediates: tracking images, one-to-one shifts, dense flow, masks
    import torch
    H, W, n = burst.height, burst.width, burst.n
    xs, tx, ty = m.debug_shifts()
    x = isa.device_copy(xs, (ty * tx, n - 1, 2), torch.float32).cpu().numpy()
    assert np.abs(x - keep["x"]).max() < 1e-3
    for i in range(1, n):
        d = m.debug(i)
        fl = isa.device_copy(d["flow"], (H, W, 2), torch.float32).cpu().numpy()
        df = np.abs(fl - keep["flow"][i]).max(axis=2)
        assert np.percentile(df, 99.9) < 1e-3 and df.max() < 0.05
        mk = isa.device_copy(d["mask"], (H // 2, W // 2, 4), torch.float32).cpu().numpy()
        dm = np.abs(mk - keep["mask"][i])[..., :3].max(axis=2)
        assert (dm > 1e-4).mean() < 1e-3
    bt = isa.device_copy(m.debug(0)["bw_track"], (H, W), torch.float32).cpu().numpy()
    assert np.abs(bt - keep["bw_track"][0]).max() < 2e-5
    m.close()


@pytest.mark.parametrize("case", ["onref", "refblock", "blocks", "ref2", "prealign", "bggr", "moving"])
def test_merge_variants_match_oracle(cuda, oracle, case):
    """Tracking strategies, reference choice, pre-alignment input, another
    Bayer layout, and an independently moving object (5 % of the frame,
    2-40 px per frame: the robustness mask rejects it where it occludes)."""
    cfa = "BGGR" if case == "bggr" else "RGGB"
    b = synthetic.make_burst(512, 384, 6, seed=33, max_shift=5, max_rot_deg=0.2, cfa=cfa, moving_object=0.05 if case == "moving" else 0.0)
    p = P.MergeParams()
    p.merge_scale = 2.0
    pre = PL.PreAlignment.zeros(b.n)
    if case == "onref":
        p.tracking_strategy = P.ONLY_ON_REFERENCE
    elif case == "refblock":
        p.tracking_strategy, p.tracking_block_size = P.ON_REFERENCE_BLOCK, 3
        pre.reference = 4
    elif case == "blocks":
        p.tracking_strategy, p.tracking_block_size = P.BLOCKS, 2
    elif case == "ref2":
        pre.reference = 2
    elif case == "prealign":
        pre.shifts = np.array([[0, 0], [3.2, -1.5], [-2.0, 4.4], [1.0, 1.0], [0.5, -0.5], [-3.0, -2.0]])
        pre.rotations = np.array([0.0, 0.1, -0.15, 0.05, 0.0, 0.2])
        pre.reference = 1
    keep = {}
    want = PL.merge_burst(b, p, lib=oracle, pre=pre, keep=keep)
    m, got = gpu_merge(b, p, pre=pre)
    image_parity(m, b, p, got, want, keep, reference=pre.reference)
    m.close()


def test_fused_and_per_frame_accumulation_are_identical(cuda, burst):
    p = P.MergeParams()
    p.merge_scale = 2.0
    m1, a = gpu_merge(burst, p, fused=True)
    m2, b = gpu_merge(burst, p, fused=False)
    np.testing.assert_array_equal(a, b)
    m1.close()
    m2.close()


def test_host_and_device_entry_points_agree(cuda, burst):
    import torch
    p = P.MergeParams()
    m, a = gpu_merge(burst, p)
    host_raw = torch.from_numpy(burst.raw.view(np.int16)).pin_memory()
    b = m.merge_host(host_raw, isa.make_info(burst))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a, b)
    m.close()


def test_bad_arguments_leave_the_context_usable(cuda, burst):
    import torch
    p = P.MergeParams()
    m = isa.Merger(burst.width, burst.height, burst.n, p)
    info = isa.make_info(burst)
    raw = to_dev(burst.raw)
    with pytest.raises(isa.IsaError):
        m.merge(raw, info, reference=7)
    bad = isa.make_info(burst)
    bad.width = burst.width + 2  # larger than the context
    out = torch.empty((burst.height, burst.width, 3), device="cuda")
    with pytest.raises(isa.IsaError):
        isa.check(isa.lib().isa_merge_burst(m.ctx, isa.vp(raw), ctypes.c_size_t(burst.width * 2), ctypes.c_size_t(raw.numel() * 2 // burst.n),
                                            burst.n, ctypes.byref(bad), None, isa.vp(out), ctypes.c_size_t(burst.width * 12), None))
    bad = isa.make_info(burst)
    bad.cfa[1] = 3
    with pytest.raises(isa.IsaError):
        m.merge(raw, bad)
    got = m.merge(raw, info)
    torch.cuda.synchronize()
    assert torch.isfinite(got).all()
    m.close()


@pytest.fixture(scope="module")
def full_burst():
    return synthetic.make_burst(6016, 4000, 20, seed=1000, max_shift=24.0, max_rot_deg=0.5, noise_a=1e-3, noise_b=8e-6, device="cuda")


def test_full_size_fused_equals_per_frame(cuda, full_burst):
    """At the benchmark size (20 x 6016 x 4000 -> 12032 x 8000): the fused
    accumulation reads every frame once and must reproduce the reference's
    frame-by-frame read-modify-write passes bit for bit."""
    import torch
    p = P.MergeParams()
    p.merge_scale = 2.0
    m1 = isa.Merger(6016, 4000, 20, p, fused_accumulate=True)
    m2 = isa.Merger(6016, 4000, 20, p, fused_accumulate=False)
    raw = to_dev(full_burst.raw)
    info = isa.make_info(full_burst)
    a = m1.merge(raw, info)
    b = m2.merge(raw, info)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert torch.isfinite(a).all()
    inner = a[16:-16, 16:-16]
    assert float(inner.min()) > -0.1 and float(inner.max()) < 1.1
    m1.close()
    m2.close()


def test_full_size_known_shift(cuda):
    """Frames that are exact integer translates of a textured frame 0 (the
    seeded blurred-noise scene of the reference's test mode, TestRawFile.cs:
    39-64; even shifts keep the CFA phase) at the full 6016 x 4000 size: LK
    converges to the translation, so round(2 * flow) is the exact 2x shift
    almost everywhere. MatchingThreshold is 0 here: the default 1.0 is an
    absolute bound on the L2 range of a 32 x 32 tile of high-passed image and
    suppresses the coarse levels on this fine-grained texture."""
    import torch
    import torch.nn.functional as F
    W, H = 6016, 4000
    g = torch.Generator(device="cuda").manual_seed(3)
    tex = F.avg_pool2d(torch.rand((1, 1, H + 64, W + 64), generator=g, device="cuda"), 5, stride=1, padding=2)[0, 0]
    tex = (tex - tex.min()) / (tex.max() - tex.min())
    shifts = [(0, 0), (6, -4), (-10, 8), (2, 14)]
    raw = torch.empty((4, H, W), dtype=torch.int16, device="cuda")
    for i, (dx, dy) in enumerate(shifts):
        t = tex[32 - dy:32 - dy + H, 32 - dx:32 - dx + W]
        raw[i] = torch.round(512 + t * 15000).to(torch.int16)
    b = synthetic.Burst(raw=np.zeros((4, 2, 2), np.uint16), cfa=(0, 1, 1, 2), black=(512.0,) * 3, white=(15871.0,) * 3, noise_a=1e-3,
                        noise_b=8e-6, shifts=np.zeros((4, 2)), rotations=np.zeros(4))
    info = isa.make_info(b)
    info.width, info.height = W, H
    p = P.MergeParams()
    p.merge_scale = 2.0
    p.matching_threshold = 0.0
    m = isa.Merger(W, H, 4, p)
    m.merge(raw, info)
    torch.cuda.synchronize()
    for i in range(1, 4):
        fl = isa.device_copy(m.debug(i)["flow"], (H, W, 2), torch.float32)[64:-64, 64:-64].reshape(-1, 2)
        want = torch.tensor(shifts[i], device="cuda", dtype=torch.float32)
        exact = (torch.round(fl * 2) == want * 2).all(dim=1).float().mean()
        assert float(exact) > 0.98, (i, float(exact))
        assert float((fl - want).abs().median()) < 1e-2
    m.close()


def test_pipeline_masks_equal_operator_masks(cuda, burst):
    """The merge computes the robustness mask from reference statistics made
    once per burst and the moved image's 3x3 means made once per frame; the
    operator entry point isa_robustness_erode evaluates every tap directly.
    Both must give the same masks bit for bit, on the pipeline's own flows."""
    import torch
    p = P.MergeParams()
    p.merge_scale = 2.0
    m = isa.Merger(burst.width, burst.height, burst.n, p)
    info = isa.make_info(burst)
    raw = to_dev(burst.raw)
    m.merge(raw, info)
    torch.cuda.synchronize()
    H, W, n = burst.height, burst.width, burst.n
    Wh, Hh = W // 2, H // 2
    maxv = max(w + b for w, b in zip(burst.white, burst.black))
    cfa = (ctypes.c_int * 4)(*burst.cfa)
    sz = ctypes.c_size_t
    frames = raw.view(n, H, W)
    half = []
    for i in range(n):
        h = torch.zeros((Hh, Wh, 3), dtype=torch.float32, device="cuda")
        isa.check(isa.lib().isa_debayer_subsample(isa.vp(frames[i]), sz(W * 2), W, H, cfa, ctypes.c_float(maxv), isa.vp(h), sz(Wh * 12), None))
        half.append(h)
    for i in range(1, n):
        d = m.debug(i)
        flow = isa.device_copy(d["flow"], (H, W, 2), torch.float32)
        want = isa.device_copy(d["mask"], (Hh, Wh, 4), torch.float32)
        got = torch.zeros_like(want)
        isa.check(isa.lib().isa_robustness_erode(isa.vp(half[0]), isa.vp(half[i]), sz(Wh * 12), Wh, Hh, isa.vp(flow), sz(W * 8), W, H,
                                                 ctypes.c_float(burst.noise_a), ctypes.c_float(burst.noise_b), ctypes.c_float(p.threshold_m),
                                                 ctypes.c_float(p.robust_s), ctypes.c_float(p.robust_t), p.erode_size, isa.vp(got), sz(Wh * 16),
                                                 None))
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"frame {i}: {(got != want).sum().item()} values differ"
    m.close()
