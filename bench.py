#!/usr/bin/env python
"""Benchmark: merged MP/s of a 20 x 24 MP Bayer burst merged at 2x on B200.

One step = the whole forward merge of one burst through libisa.so
(isa_merge_burst: tracking images, 4-level tile alignment over all 190 frame
pairs with the least-squares shift solve, kernel parameters, 3 LK
iterations and the robustness mask per frame, kernel-weighted accumulation,
normalisation). Workload: 20 frames of 6016 x 4000 RGGB uint16 (14-bit,
black 512), shifts +-24 px, rotation +-0.5 deg, noise a = 1e-3, b = 8e-6,
merged over the whole frame at scale 2.0 into a 12032 x 8000 float32 RGB
image. Synthetic, seeded, generated on the GPU before timing.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun): every rank merges its own burst (weak scaling, no
collective on the data path); the step time is the max over ranks.
`--impl reference` times the reference's own kernel bodies compiled for the
host (oracle/_ref, FP32, OpenMP on all cores) on a bounded sample burst of
the same statistics; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(width=6016, height=4000, frames=20, max_shift=24.0, max_rot_deg=0.5, noise_a=1e-3, noise_b=8e-6, scale=2.0)
# the host sample of the reference's kernels, for both the cpu_baseline leg and every `--impl reference` step: 20 frames
# of 1024x768 with the headline workload's statistics merged at 2x (about 8 s on 16 host cores; MP/s is per output pixel,
# so the sample's rate stands for the 20 x 6016x4000 workload's)
SAMPLE = dict(width=1024, height=768)
REF_STEP = SAMPLE
METRIC = "merged MP/s"
UNIT = "MP/s"


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the accumulation kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "accumulate_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload_burst(rank, device, width=None, height=None):
    from imagestackalignator_b200 import synthetic
    w = width or WORKLOAD["width"]
    h = height or WORKLOAD["height"]
    return synthetic.make_burst(w, h, WORKLOAD["frames"], seed=burst_seed(rank), max_shift=WORKLOAD["max_shift"],
                                max_rot_deg=WORKLOAD["max_rot_deg"], noise_a=WORKLOAD["noise_a"], noise_b=WORKLOAD["noise_b"],
                                device=device)


def burst_seed(rank):
    """Each rank merges its own burst: seeds differ per rank, identical across runs."""
    return 1000 + rank


def reduce_max(x, dist, device):
    """The slowest rank's value (step times are reported as the max over ranks)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, out_mp_per_rank, ms_per_step):
    """Whole-job throughput: every rank's output megapixels over the slowest rank's step time."""
    return world * out_mp_per_rank / (ms_per_step / 1e3)


def merge_params():
    from imagestackalignator_b200 import params as P
    p = P.MergeParams()
    p.merge_scale = WORKLOAD["scale"]
    return p


_SAMPLE_BURSTS = {}


def cpu_reference_run(width, height, threads):
    """One merge of a sample burst by the reference kernels on the host (FP32, OpenMP); the burst is made once."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pipeline as PL
    if (width, height) not in _SAMPLE_BURSTS:
        _SAMPLE_BURSTS[(width, height)] = make_workload_burst(0, "cpu", width, height)
    b = _SAMPLE_BURSTS[(width, height)]
    lib = PL.StageLib("ref32")
    lib.set_threads(threads)
    t0 = time.perf_counter()
    r = PL.merge_burst(b, merge_params(), lib=lib)
    dt = time.perf_counter() - t0
    out_px = r.image.shape[0] * r.image.shape[1]
    return out_px, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    w, h = REF_STEP["width"], REF_STEP["height"]
    for _ in range(args.warmup):
        cpu_reference_run(w, h, threads)
    times = []
    out_px = 0
    for _ in range(args.steps):
        out_px, dt = cpu_reference_run(w, h, threads)
        times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    value = out_px / 1e6 / (ms / 1e3)
    sample = f"{WORKLOAD['frames']} frames of {w}x{h} RGGB (config statistics) merged at 2x -> {2 * w}x{2 * h}, per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "20-frame RGGB burst merged at 2x (reference kernels on the host, bounded sample)", "frames": WORKLOAD["frames"],
                   "sample": f"{w}x{h}", "stands_for": f"{WORKLOAD['frames']} x {WORKLOAD['width']}x{WORKLOAD['height']} merged at 2x",
                   "same_sample_as_cpu_baseline": True, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


ADJ = dict(width=4000, height=3000, frames=10, scale=1.5)  # the differentiable-merge workload (10 x 4000x3000 at 1.5x)


def adjoint_ratio(args):
    """Forward merge vs forward + adjoint (isa_merge_backward) of an L2 loss on
    the differentiable-merge workload, device time per call, same warm-up and
    step counts as the main measurement."""
    import torch
    from imagestackalignator_b200 import isa, params as P, synthetic
    W, H, n = ADJ["width"], ADJ["height"], ADJ["frames"]
    b = synthetic.make_burst(W, H, n, seed=2000, max_shift=WORKLOAD["max_shift"], max_rot_deg=WORKLOAD["max_rot_deg"],
                             noise_a=WORKLOAD["noise_a"], noise_b=WORKLOAD["noise_b"], device="cuda")
    p = merge_params()
    p.merge_scale = ADJ["scale"]
    m = isa.Merger(W, H, n, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(b.raw.view(np.int16)).cuda()
    out = m.merge(raw, info)
    target = (0.9 * out + 0.03).contiguous()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    fwd = timed(lambda: m.merge(raw, info, out))
    both = timed(lambda: m.backward(raw, info, target, out=out))
    m.close()
    # sample mode BILINEAR: the same, plus the gradient of every frame's tile flow (isa_merge_backward_tiles)
    pb = merge_params()
    pb.merge_scale = ADJ["scale"]
    pb.sample_mode = P.SAMPLE_BILINEAR
    mb = isa.Merger(W, H, n, pb)
    fwd_b = timed(lambda: mb.merge(raw, info, out))
    both_b = timed(lambda: mb.backward_tiles(raw, info, target, out=out))
    mb.close()
    return {"workload": f"{n}x{W}x{H} merged at {ADJ['scale']}x, L2 loss, gradients of the 8 merge parameters", "fwd_ms": fwd,
            "fwd_adj_ms": both, "ratio": both / fwd,
            "bilinear": {"workload": "sample mode BILINEAR, gradients of the 8 merge parameters and of every frame's tile flow",
                         "fwd_ms": fwd_b, "fwd_adj_tiles_ms": both_b, "ratio": both_b / fwd_b}}


def param_fit(width, height, frames, steps, moving_object=0.0, max_shift=None, seed=3000):
    """Adam on the eight merge parameters (isa_merge_backward), in log space
    from the reference defaults, fitting the merge at scale 1 to the clean
    scene of the reference frame (the synthetic generator keeps it). Loss and
    PSNR over the output pixels inside a 32 px margin whose smallest weight
    sum is at least 0.05; PSNR against the scene before and after the fit."""
    import torch
    from imagestackalignator_b200 import fit, isa, params as P, synthetic
    b = synthetic.make_burst(width, height, frames, seed=seed, max_shift=max_shift or WORKLOAD["max_shift"],
                             max_rot_deg=WORKLOAD["max_rot_deg"], noise_a=WORKLOAD["noise_a"], noise_b=WORKLOAD["noise_b"], device="cuda",
                             keep_truth=True, moving_object=moving_object)
    p = P.MergeParams()
    p.merge_scale = 1.0
    m = isa.Merger(width, height, frames, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(b.raw.view(np.int16)).cuda()
    truth = torch.from_numpy(b.truth.astype(np.float32)).cuda().contiguous()
    out = m.merge(raw, info).clone()
    wsum = isa.device_copy(m.debug(0)["wsum"], (height, width, 3), torch.float32)
    om = (wsum.min(dim=2).values >= 0.05).float()
    om[:32] = 0
    om[-32:] = 0
    om[:, :32] = 0
    om[:, -32:] = 0
    om = om.contiguous()
    npx = float(om.sum())

    def psnr(img):
        mse = float((om[..., None] * (img - truth) ** 2).sum()) / (3 * npx)
        return 10 * np.log10(1.0 / mse)

    base = np.array([getattr(p, k) for k in fit.NAMES], np.float64)
    psnr0 = psnr(out)
    torch.cuda.synchronize()
    t0 = time.time()
    theta, losses = fit.adam_fit(fit.merger_grad_fn(m, p, raw, info, truth, weight=om, out=out), base, steps)
    m.set_params(fit.params_of(p, theta))
    fitted = m.merge(raw, info, out).clone()
    torch.cuda.synchronize()
    dt = time.time() - t0
    res = {"workload": f"{frames}x{width}x{height} merged at 1x" + (f", moving object {moving_object:.0%} of the frame" if moving_object else ""),
           "steps": steps, "loss_first": losses[0], "loss_last": losses[-1], "psnr_before_db": psnr0, "psnr_after_db": psnr(fitted),
           "ms_per_step": 1000 * dt / steps, "params_after": {k: float(v) for k, v in zip(fit.NAMES, theta)}}
    m.close()
    return res


BATCH = dict(width=2048, height=1536, frames=8, bursts=16, contexts=4)  # many small bursts (phone-sized) merged at 2x


def batch_throughput(args):
    """Many small bursts: one context on one stream (isa_merge_burst per burst)
    against isa_merge_batch over several contexts and streams, device time for
    the whole set of bursts, same warm-up and step counts as the main line."""
    import torch
    from imagestackalignator_b200 import isa, synthetic
    W, H, n, nb, nc = BATCH["width"], BATCH["height"], BATCH["frames"], BATCH["bursts"], BATCH["contexts"]
    p = merge_params()
    mergers = [isa.Merger(W, H, n, p) for _ in range(nc)]
    Wo, Ho = mergers[0].output_size(W, H)
    items = []
    for i in range(nb):
        b = synthetic.make_burst(W, H, n, seed=3000 + i, max_shift=WORKLOAD["max_shift"], max_rot_deg=WORKLOAD["max_rot_deg"],
                                 noise_a=WORKLOAD["noise_a"], noise_b=WORKLOAD["noise_b"], device="cuda")
        items.append(dict(raw=torch.from_numpy(b.raw.view(np.int16)).cuda(), info=isa.make_info(b),
                          out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda")))
    main = torch.cuda.current_stream()
    streams = [torch.cuda.Stream() for _ in range(nc)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def sequential():
        for it in items:
            mergers[0].merge(it["raw"], it["info"], it["out"], stream=main)

    def batched():
        for s in streams:
            s.wait_stream(main)
        st = isa.merge_batch(mergers, items, streams)
        if any(st):
            raise RuntimeError(f"isa_merge_batch status {st}")
        for s in streams:
            main.wait_stream(s)

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0.record(main)
        for _ in range(args.steps):
            fn()
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    seq = timed(sequential)
    bat = timed(batched)
    for m in mergers:
        m.close()
    mp = nb * Wo * Ho / 1e6
    return {"workload": f"{nb} bursts of {n}x{W}x{H} merged at 2x", "contexts": nc, "sequential_ms": seq, "batched_ms": bat,
            "sequential_mp_s": mp / (seq / 1e3), "batched_mp_s": mp / (bat / 1e3), "batched_bursts_s": nb / (bat / 1e3)}


UNEVEN = dict(bursts=64, contexts=4, frames=(4, 30), mp=(2.0, 12.0), seed=5000)  # the uneven batch: sizes, counts, CFA, depth, scale


def uneven_specs():
    """64 bursts: frame counts uniform 4-30, frame areas uniform 2-12 MP at 4:3
    or 3:2 (sides multiples of 16), CFA RGGB / BGGR / GRBG, 12 or 14 bits,
    merge scale 1 or 2; seeded."""
    rng = np.random.default_rng(UNEVEN["seed"])
    specs = []
    for i in range(UNEVEN["bursts"]):
        n = int(rng.integers(UNEVEN["frames"][0], UNEVEN["frames"][1] + 1))
        area = rng.uniform(*UNEVEN["mp"]) * 1e6
        aspect = (4 / 3, 3 / 2)[int(rng.integers(2))]
        H = max(64, int(round(np.sqrt(area / aspect) / 16)) * 16)
        W = max(64, int(round(H * aspect / 16)) * 16)
        specs.append(dict(n=n, W=W, H=H, cfa=("RGGB", "BGGR", "GRBG")[int(rng.integers(3))], bits=(12, 14)[int(rng.integers(2))],
                          scale=(1.0, 2.0)[int(rng.integers(2))], seed=UNEVEN["seed"] + i))
    return specs


def uneven_batch(args):
    """The uneven batch: 64 bursts of uneven sizes, frame counts, CFA layouts,
    bit depths and merge scales. Sequential (one context, one stream, burst by
    burst) against isa_merge_batch over several contexts and streams, both
    with the launch shapes of the project's autotuner (imagestackalignator_b200
    .tune, JSON cache), and the batch without them; device time for the set."""
    import torch
    from imagestackalignator_b200 import isa, params as P, synthetic, tune
    specs = uneven_specs()
    mw, mh, mn = max(s["W"] for s in specs), max(s["H"] for s in specs), max(s["n"] for s in specs)
    p = merge_params()
    p.merge_scale = 2.0
    mergers = [isa.Merger(mw, mh, mn, p) for _ in range(UNEVEN["contexts"])]
    items, mp = [], 0.0
    for sp in specs:
        white = (1 << sp["bits"]) - 1
        b = synthetic.make_burst(sp["W"], sp["H"], sp["n"], seed=sp["seed"], max_shift=WORKLOAD["max_shift"], max_rot_deg=WORKLOAD["max_rot_deg"],
                                 noise_a=WORKLOAD["noise_a"], noise_b=WORKLOAD["noise_b"], black=white // 32, white_max=white, cfa=sp["cfa"],
                                 device="cuda")
        q = P.MergeParams(**vars(p))
        q.merge_scale = sp["scale"]
        Wo, Ho = isa.output_size(isa.make_params(q), sp["W"], sp["H"])
        items.append(dict(raw=torch.from_numpy(b.raw.view(np.int16)).cuda(), info=isa.make_info(b), params=q,
                          out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda")))
        mp += Wo * Ho / 1e6
    main = torch.cuda.current_stream()
    streams = [torch.cuda.Stream() for _ in mergers]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run(ms, sts):
        for s in sts:
            s.wait_stream(main)
        st = isa.merge_batch(ms, items, sts)
        if any(st):
            raise RuntimeError(f"isa_merge_batch status {st}")
        for s in sts:
            main.wait_stream(s)

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0.record(main)
        for _ in range(args.steps):
            fn()
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    untuned = timed(lambda: run(mergers, streams))
    t0 = time.time()
    entries = tune.tune(mergers[0], items)
    tune_s = time.time() - t0
    for m in mergers:
        m.set_tuning(entries)
    seq = timed(lambda: run(mergers[:1], [main]))
    bat = timed(lambda: run(mergers, streams))
    # the same batch captured once as a CUDA graph and replayed (one host launch per batch)
    origin = torch.cuda.Stream()
    graph = isa.BatchGraph(mergers, items, streams, origin)

    def replay():
        origin.wait_stream(main)
        graph.launch(origin)
        main.wait_stream(origin)

    gr = timed(replay)
    graph.close()
    for m in mergers:
        m.close()
    frames = sum(s["n"] for s in specs)
    return {"workload": f"{len(specs)} bursts, {frames} frames of 2-12 MP (4:3, 3:2), 4-30 frames, RGGB/BGGR/GRBG, 12/14-bit, scale 1 or 2",
            "output_mp": mp, "contexts": len(mergers), "sequential_ms": seq, "batched_ms": bat, "batched_untuned_ms": untuned,
            "graph_ms": gr, "graph_mp_s": mp / (gr / 1e3), "graph_bursts_s": len(specs) / (gr / 1e3),
            "sequential_mp_s": mp / (seq / 1e3), "batched_mp_s": mp / (bat / 1e3), "batched_bursts_s": len(specs) / (bat / 1e3),
            "sequential_bursts_s": len(specs) / (seq / 1e3), "tuning_classes": len({tune.burst_class(e["width"], e["height"], 0) for e in entries}),
            "tuning_s": tune_s}


LARGE = dict(width=6016, height=4000, frames=50, max_shift=32.0, max_rot_deg=0.5, moving_object=0.05, object_step=(2.0, 40.0))


def large_motion_throughput(args):
    """The large burst with local motion: 50 frames of 6016x4000 RGGB 14-bit,
    global shifts of +-32 px, and a rigid textured object covering 5 % of the
    frame that moves 2-40 px per frame on its own path; merged at 2x with the
    Full strategy (1,225 frame pairs). Device time per merge, frames resident."""
    import torch
    from imagestackalignator_b200 import isa, synthetic
    W, H, n = LARGE["width"], LARGE["height"], LARGE["frames"]
    b = synthetic.make_burst(W, H, n, seed=4000, max_shift=LARGE["max_shift"], max_rot_deg=LARGE["max_rot_deg"], noise_a=WORKLOAD["noise_a"],
                             noise_b=WORKLOAD["noise_b"], device="cuda", moving_object=LARGE["moving_object"], object_step=LARGE["object_step"])
    raw = torch.from_numpy(b.raw.view(np.int16)).cuda()
    info = isa.make_info(b)
    m = isa.Merger(W, H, n, merge_params())
    Wo, Ho = m.output_size(W, H)
    out = torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda")
    main = torch.cuda.current_stream()
    steps = max(1, min(args.steps, 3))
    for _ in range(max(1, min(args.warmup, 2))):
        m.merge(raw, info, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(steps):
        m.merge(raw, info, out)
    e1.record(main)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    stages = m.stage_times()
    m.close()
    names = ["tracking_images", "tile_alignment", "kernel_params", "lk_and_robustness", "accumulation", "finalize"]
    return {"workload": f"{n}x{W}x{H} RGGB, shifts +-{LARGE['max_shift']:.0f} px, a 5 % object moving 2-40 px per frame, merged at 2x",
            "pairs": n * (n - 1) // 2, "steps": steps, "ms_per_burst": ms, "mp_s": Wo * Ho / 1e6 / (ms / 1e3),
            "stages_ms": dict(zip(names, stages))}


def post_throughput(args, merged):
    """Colour/tone post-processing (isa_postprocess, the SaveAs16BitTiff chain)
    of the merged image to uint16 RGB: device time per call, HBM roofline."""
    import torch
    from imagestackalignator_b200 import isa
    Ho, Wo, _ = merged.shape
    lx = np.float32(np.round(np.arange(256) / 255.0, 9))
    ly = np.float32(np.clip(lx + 0.12 * np.sin(2 * np.pi * lx) / (2 * np.pi), 0, 1))
    cam = np.array([[0.62, 0.24, 0.10], [0.27, 0.69, 0.04], [0.03, 0.12, 0.68]])
    t1, t2 = isa.color_twists(cam)
    pp, keep = isa.post_params((0, 0, Wo, Ho), [1.0, 1.0, 1.0], t1, t2, lx, ly, 0.0)
    out16 = torch.empty((Ho, Wo, 3), dtype=torch.int16, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(max(1, args.warmup)):
        isa.postprocess(merged, pp, isa.POST_RGB16, out16)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        isa.postprocess(merged, pp, isa.POST_RGB16, out16)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    alg = Wo * Ho * (12 + 6)
    peak, kind = measured_peak()
    gbs = alg / (ms / 1e3) / 1e9
    return {"workload": f"{Wo}x{Ho} float3 -> uint16 RGB (clamp, 2 colour twists, 256-level cubic LUT, exposure, sRGB gamma)",
            "ms": ms, "mp_s": Wo * Ho / 1e6 / (ms / 1e3), "algorithmic_bytes": alg, "achieved_gbs": gbs, "frac": gbs / peak,
            "peak_source": f"{kind} hbm_gbs",
            "l2": f"input {Wo * Ho * 12 / 1e9:.2f} GB {'larger' if Wo * Ho * 12 > 126e6 else 'smaller'} than the 126 MB L2"}


def raw_decode_throughput(args, frame):
    """PEF raw decoding (isa_pef_decode) of one frame of the workload,
    compressed in the reference's stream layout: device time per frame
    (one launch sequence, no host round trips), with
    the restated reference decoder on one host core as its CPU baseline."""
    import torch
    from imagestackalignator_b200 import isa, synthetic
    H, W = frame.shape
    code, lens = synthetic.pef_code_book()
    stream = synthetic.pef_stream(frame, code, lens)
    table = isa.pef_huff_table(synthetic.pef_maker_note(code, lens))
    d = torch.from_numpy(stream).cuda()
    out = torch.empty((H, W), dtype=torch.int16, device="cuda")
    scratch = torch.empty(isa.lib().isa_pef_decode_scratch(ctypes.c_size_t(stream.size), W, H), dtype=torch.uint8, device="cuda")
    stream_t = torch.cuda.current_stream()
    for _ in range(max(1, args.warmup)):
        isa.pef_decode(d, table, W, H, out, scratch)
    torch.cuda.synchronize()
    exact = bool(np.array_equal(out.cpu().numpy().view(np.uint16), frame))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream_t)
    for _ in range(args.steps):
        isa.pef_decode(d, table, W, H, out, scratch)
    e1.record(stream_t)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    res = {"workload": f"one {W}x{H} 14-bit frame of the burst, {stream.size / 1e6:.1f} MB compressed ({stream.size * 8 / frame.size:.2f} bits/px)",
           "ms": ms, "mp_s": W * H / 1e6 / (ms / 1e3), "compressed_gb_s": stream.size / 1e9 / (ms / 1e3),
           "exact": exact, "cpu_baseline": None}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import raw as R  # the restated reference decoder (PEFFile.cs:35-111), one host core
        t0 = time.perf_counter()
        R.decode(stream, table, W, H)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"mp_s": W * H / 1e6 / dt, "cores": 1, "kind": "port", "sample": f"the same {W}x{H} stream, {dt:.2f} s"}
    return res


def dng_decode_throughput(args, frame):
    """DNG raw decoding (isa_dng_decode) of one frame of the workload stored
    as 256 x 256 lossless-JPEG tiles (two interleaved components, predictor
    1): time per frame through the entry point (host header parsing, the
    parallel decoder, synchronised; file bytes already on the device), with
    the restated reference reader on one host core as its CPU baseline."""
    import torch
    from imagestackalignator_b200 import isa, synthetic
    H, W = frame.shape
    f, offs, cnts = synthetic.dng_tiled_file(frame)
    dev = torch.from_numpy(f).cuda()
    kw = dict(tiled=True, tile_w=256, tile_h=256, file_dev=dev)
    scratch = torch.empty(isa.dng_decode_scratch(f, W, H, offs, cnts, tiled=True, tile_w=256, tile_h=256), dtype=torch.uint8, device="cuda")
    out = torch.empty((H, W), dtype=torch.int16, device="cuda")
    for _ in range(max(1, args.warmup)):
        isa.dng_decode(f, W, H, offs, cnts, scratch=scratch, out=out, **kw)
    torch.cuda.synchronize()
    exact = bool(np.array_equal(out.cpu().numpy().view(np.uint16), frame))
    path = isa.dng_decode_path()
    stream_t = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream_t)
    for _ in range(args.steps):
        isa.dng_decode(f, W, H, offs, cnts, scratch=scratch, out=out, **kw)
    e1.record(stream_t)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    res = {"workload": f"one {W}x{H} 14-bit frame as {len(offs)} lossless-JPEG tiles of 256x256, {f.size / 1e6:.1f} MB", "ms": ms,
           "mp_s": W * H / 1e6 / (ms / 1e3), "compressed_gb_s": f.size / 1e9 / (ms / 1e3), "exact": exact,
           "decoder": {1: "parallel (candidate-start maps)", 0: "per-part reader"}.get(path, "none"), "cpu_baseline": None}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import raw as R  # the restated reference reader (DNGFile.cs:40-600), one host core
        t0 = time.perf_counter()
        R.dng_decode(f, W, H, offs, cnts, tiled=True, tile_w=256, tile_h=256)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"mp_s": W * H / 1e6 / dt, "cores": 1, "kind": "port", "sample": f"the same file, {dt:.2f} s"}
    return res


def files_throughput(args, burst, merger, out):
    """The reference's flow from raw files, end to end: the burst's frames as
    DNG files (host bytes), each opened (isa_dng_open, colour spec, levels),
    copied to the device and decoded (isa_dng_decode), then merged at 2x
    (isa_merge_burst) and the image read back; everything from the files'
    host bytes to the host image inside the timed region."""
    import torch
    from imagestackalignator_b200 import isa, synthetic
    n, H, W = burst.raw.shape
    # the files (untimed): 256 x 256 tiles, the burst's noise profile, a neutral white point
    files = [synthetic.dng_file(np.ascontiguousarray(burst.raw[f]), tile=256, noise=[burst.noise_a, burst.noise_b],
                                color=dict(as_shot_neutral=[1.0, 1.0, 1.0]), threads=os.cpu_count() or 1)[0] for f in range(n)]
    hosts = [torch.from_numpy(f).pin_memory() for f in files]
    devs = [torch.empty(f.size, dtype=torch.uint8, device="cuda") for f in files]
    copy_stream = torch.cuda.Stream()
    frames = torch.empty((n, H, W), dtype=torch.int16, device="cuda")
    scratches = [torch.empty(isa.dng_decode_scratch(f, W, H, **isa.dng_open(f)["layout"]), dtype=torch.uint8, device="cuda") for f in files]
    Ho, Wo = out.shape[0], out.shape[1]
    host_out = torch.empty((Ho, Wo, 3), dtype=torch.float32).pin_memory()

    def step():
        # every file's bytes go to the device on a side stream, each decode waiting only for its own file
        copied = []
        with torch.cuda.stream(copy_stream):
            for i in range(n):
                devs[i].copy_(hosts[i], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(copy_stream)
                copied.append(ev)
        info = None
        calls = []
        for i, f in enumerate(files):   # every decode enqueued (isa_dng_decode_begin), then one wait (isa_dng_decode_finish)
            d = isa.dng_open(f)
            c2p, cw, _ = isa.dng_color_spec(**d["color"])
            lv = isa.dng_levels(camera_white=cw, **d["levels"])
            torch.cuda.current_stream().wait_event(copied[i])
            kw = dict(black_h=lv["black_h"], black_v=lv["black_v"], file_dev=devs[i], scratch=scratches[i], out=frames[i], **d["layout"])
            isa.dng_decode(f, W, H, phase="begin", **kw)
            calls.append((f, kw))
            info = lv["info"] if i == 0 else info
        for f, kw in calls:
            isa.dng_decode(f, W, H, phase="finish", **kw)
        merger.merge(frames, info, out)
        host_out.copy_(out, non_blocking=True)
        torch.cuda.synchronize()

    step()
    exact = bool(np.array_equal(frames.cpu().numpy().view(np.uint16), burst.raw))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    return {"workload": f"{n} DNG files of {W}x{H} (256x256 lossless-JPEG tiles, {sum(f.size for f in files) / 1e6:.0f} MB) -> "
                        f"{Wo}x{Ho} RGB merged at 2x, host bytes in, host image out",
            "value": Wo * Ho / 1e6 / dt, "unit": UNIT, "ms": dt * 1e3, "frames_exact": exact,
            "h2d_bytes_per_step": int(sum(f.size for f in files)), "d2h_bytes_per_step": int(Wo * Ho * 12),
            "timing": "host wall clock around each synchronised step (all decodes enqueued, then one wait for their flags)"}


def run_ours(args):
    import torch
    from imagestackalignator_b200 import isa

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    W, H, n = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["frames"]
    burst = make_workload_burst(rank, "cuda")
    info = isa.make_info(burst)
    merger = isa.Merger(W, H, n, merge_params(), fused_accumulate=not args.per_frame)
    Wo, Ho = merger.output_size(W, H)
    raw = torch.from_numpy(burst.raw.view(np.int16)).cuda()
    out = torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        merger.merge(raw, info, out)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        merger.merge(raw, info, out)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_total = e0.elapsed_time(e1)
    stages = merger.stage_times()
    launches = merger.launch_count() * args.steps
    clocks = sampler.stop()
    ms_total = reduce_max(ms_total, dist, "cuda")
    ms = ms_total / args.steps
    out_mp = Wo * Ho / 1e6
    value = job_value(world, out_mp, ms)

    # end to end through the C ABI with host buffers (H2D of the frames and D2H of the image inside the timed region)
    e2e = None
    if not args.no_e2e:
        host_raw = torch.from_numpy(burst.raw.view(np.int16)).pin_memory()
        host_out = torch.empty((Ho, Wo, 3), dtype=torch.float32).pin_memory()
        merger.merge_host(host_raw, info, host_out)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            merger.merge_host(host_raw, info, host_out)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        t_e2e = reduce_max(e0.elapsed_time(e1), dist, "cuda")
        e2e = {"value": job_value(world, out_mp, t_e2e / args.steps), "unit": UNIT, "h2d_bytes_per_step": int(burst.raw.nbytes),
               "d2h_bytes_per_step": int(Wo * Ho * 12)}

    peak, peak_kind = measured_peak()
    # accumulation kernel: algorithmic bytes per output pixel (fused, all frames in one launch):
    # n * (2 + 8 + 4) / s^2 (raw, flow, mask per frame) + 16 / s^2 (kernel parameters) + 24 (write-only sums)
    s = WORKLOAD["scale"]
    if args.per_frame:
        bpp = 2 / s ** 2 + 8 / s ** 2 + 16 / (4 * s ** 2) + 16 / s ** 2 + 48
        launches_acc = n
    else:
        bpp = n * (2 + 8 + 4) / s ** 2 + 16 / s ** 2 + 24
        launches_acc = 1
    acc_ms = stages[4] / launches_acc if len(stages) > 4 else None
    alg_bytes = bpp * Wo * Ho
    achieved = alg_bytes / (acc_ms / 1e3) / 1e9 if acc_ms else None
    tr = profile_traffic()
    roofline = {"kernel": f"k_accumulate_x2 (fused, {n} frames)" if not args.per_frame else "k_accumulate_x2 (one frame)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg_bytes,
                "traffic": tr.get("dram_bytes_per_launch") if tr else None}
    if not args.per_frame and acc_ms:
        # the reference's layout: one pass per frame reading raw, flow, mask and kernel and reading and
        # writing the float3 sums, n passes in the time of the fused launch (which is issue-bound, not HBM-bound)
        ref_bytes = ((2 + 8 + 16 / 4 + 16) / s ** 2 + 48) * Wo * Ho * n
        ref_gbs = ref_bytes / (stages[4] / 1e3) / 1e9
        roofline["reference_layout"] = {"bytes_per_step": ref_bytes, "achieved": ref_gbs, "frac": ref_gbs / peak,
                                        "note": "the per-frame passes of the reference moved in the fused kernel's time"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        px, dt = cpu_reference_run(SAMPLE["width"], SAMPLE["height"], threads)
        cpu = {"value": px / 1e6 / dt, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"{WORKLOAD['frames']} frames of {SAMPLE['width']}x{SAMPLE['height']} (same statistics) merged at 2x by the "
                         f"reference kernels compiled for the host (FP32, OpenMP), {dt:.1f} s wall"}
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = adjoint_ratio(args)
    uneven = None
    if rank == 0 and world == 1 and not args.no_uneven:
        uneven = uneven_batch(args)
    fit = None
    if rank == 0 and world == 1 and not args.no_fit:
        fit = param_fit(ADJ["width"], ADJ["height"], ADJ["frames"], 200)
    fit_large = None
    if rank == 0 and world == 1 and args.fit_large:
        fit_large = param_fit(LARGE["width"], LARGE["height"], LARGE["frames"], args.fit_large, moving_object=LARGE["moving_object"],
                              max_shift=LARGE["max_shift"], seed=4000)
    post = None
    if rank == 0 and world == 1 and not args.no_post:
        post = post_throughput(args, out)
    rawdec = None
    if rank == 0 and world == 1 and not args.no_raw:
        rawdec = raw_decode_throughput(args, np.ascontiguousarray(burst.raw[1]))
    dngdec = None
    if rank == 0 and world == 1 and not args.no_raw:
        dngdec = dng_decode_throughput(args, np.ascontiguousarray(burst.raw[1]))
    files = None
    if rank == 0 and world == 1 and not args.no_raw and not args.no_files:
        try:
            files = files_throughput(args, burst, merger, out)
        except Exception as exc:  # an optional key: report, keep the line
            files = {"error": f"{type(exc).__name__}: {exc}"}
    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        batch = batch_throughput(args)
    large = None
    if rank == 0 and world == 1 and not args.no_large:
        large = large_motion_throughput(args)
    names = ["tracking_images", "tile_alignment", "kernel_params", "lk_and_robustness", "accumulation", "finalize"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene, bicubic motion, Poisson-Gaussian noise; BASELINE config 1 statistics)",
        "config": {"workload": f"{n}x{W}x{H} RGGB u16 burst merged at 2x -> {Wo}x{Ho} RGB f32 (whole frame)", "frames": n,
                   "frame_size": f"{W}x{H}", "output": f"{Wo}x{Ho}", "pairs": n * (n - 1) // 2, "levels": 4, "lk_iterations": 3,
                   "accumulation": "per-frame" if args.per_frame else "fused",
                   "l2": f"inputs larger than L2 (raw frames {burst.raw.nbytes / 1e6:.0f} MB, 126 MB L2)",
                   "parallelism": f"{world} independent bursts" if world > 1 else "single GPU"},
        "stages_ms": dict(zip(names, stages)), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "fwd_adjoint": adjoint, "param_fit": fit, "param_fit_large": fit_large, "uneven_batch": uneven, "batch": batch, "large_local_motion": large, "postprocess": post, "raw_decode": rawdec, "dng_decode": dngdec, "dng_files_e2e": files,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    merger.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--per-frame", action="store_true", help="accumulate frame by frame (reference layout) instead of fused")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward+adjoint timing")
    ap.add_argument("--no-fit", action="store_true", help="skip the 200-step parameter fit on the differentiable-merge burst")
    ap.add_argument("--no-uneven", action="store_true", help="skip the 64 uneven bursts (sequential vs batched, autotuned shapes)")
    ap.add_argument("--fit-large", type=int, default=0, help="Adam steps of the parameter fit on the 50-frame burst with local motion (0: none)")
    ap.add_argument("--no-batch", action="store_true", help="skip the many-small-bursts timing")
    ap.add_argument("--no-large", action="store_true", help="skip the 50-frame burst with local motion")
    ap.add_argument("--no-post", action="store_true", help="skip the colour/tone post-processing timing")
    ap.add_argument("--no-raw", action="store_true", help="skip the PEF and DNG raw-decoding timings")
    ap.add_argument("--no-files", action="store_true", help="skip the DNG-files-to-image end-to-end timing")
    ap.add_argument("--size", default=None, help="WxH override for profiling runs on a smaller burst (not a bench line)")
    ap.add_argument("--frames", type=int, default=None, help="frame-count override for profiling runs (not a bench line)")
    args = ap.parse_args()
    if args.size:
        w, h = args.size.lower().split("x")
        WORKLOAD["width"], WORKLOAD["height"] = int(w), int(h)
    if args.frames:
        WORKLOAD["frames"] = args.frames
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
