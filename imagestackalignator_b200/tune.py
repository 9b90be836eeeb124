"""Launch-shape autotuner for batches of uneven bursts.

The shapes it chooses are the runtime knobs of isa_ctx_set_tuning: the rows
per CTA strip of the LK iteration (flow.cu k_lk_stream) and the thread block
of the accumulation at scales other than 2 and in sample mode BILINEAR
(merge.cu k_accumulate). Neither changes the order of any sum, so the merged
images do not depend on them. Bursts are grouped into classes (merge scale,
aspect ratio, frame area rounded to 2 MP); for one burst of each class every
candidate is timed on the device (CUDA events, after a warm-up merge) by
coordinate search (strip rows first, then the block); a shape replaces the
library's own choice only when it is at least 3 % faster, and the winner
applies to every frame size of the class. Results are cached as JSON keyed by class
and device name, so a later run on the same kind of GPU reuses them.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Optional

LK_ROWS = (0, 32, 48, 64, 96, 128)
ACC_BLOCKS = ((0, 0), (32, 4), (64, 4), (16, 16), (128, 2))
MARGIN = 0.03  # a shape replaces the library's choice only when at least this much faster


def default_cache_path() -> str:
    return os.environ.get("ISA_TUNING_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "imagestackalignator_b200", "tuning.json")


def burst_class(width: int, height: int, scale: float) -> str:
    aspect = "3:2" if abs(width / height - 1.5) < abs(width / height - 4 / 3) else "4:3"
    return f"s{scale:g}-{aspect}-{int(round(width * height / 2e6)) * 2}MP"


def _device_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def _time_merge(merger, item, entry, reps: int) -> float:
    import torch
    from . import isa
    merger.set_tuning([entry])
    st = isa.merge_batch([merger], [item])  # warm-up (and a check that the shapes run)
    if any(st):
        raise RuntimeError(f"merge failed with tuning {entry}: {st}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        isa.merge_batch([merger], [item])
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _pick(candidates, cost):
    """The first candidate (the library's own choice) unless another is at
    least MARGIN faster: differences within run-to-run noise keep the default."""
    t = [cost(c) for c in candidates]
    best = min(range(len(t)), key=lambda i: t[i])
    return candidates[best] if t[best] < (1.0 - MARGIN) * t[0] else candidates[0]


def tune(merger, items: List[dict], cache_path: Optional[str] = None, reps: int = 3) -> List[Dict[str, int]]:
    """Tuning entries (isa_ctx_set_tuning dicts) for every frame size of `items`
    (isa.merge_batch burst dicts; `params` gives a burst's merge scale), timed on
    `merger`'s context and cached in `cache_path` (JSON)."""
    path = cache_path or default_cache_path()
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        cache = {}
    dev = _device_name()
    classes: Dict[str, dict] = {}
    sizes: Dict[str, set] = {}
    for it in items:
        n, H, W = it["raw"].shape
        scale = float(it["params"].merge_scale) if it.get("params") is not None else 0.0
        c = burst_class(W, H, scale)
        classes.setdefault(c, it)
        sizes.setdefault(c, set()).add((W, H))
    entries = []
    changed = False
    for c, it in classes.items():
        key = f"{dev}|{c}"
        if key not in cache:
            n, H, W = it["raw"].shape
            best_rows = _pick(LK_ROWS, lambda r: _time_merge(merger, it, dict(width=W, height=H, lk_strip_rows=r), reps))
            best_blk = _pick(ACC_BLOCKS, lambda b: _time_merge(merger, it, dict(width=W, height=H, lk_strip_rows=best_rows,
                                                                                   acc_block_x=b[0], acc_block_y=b[1]), reps))
            cache[key] = dict(lk_strip_rows=best_rows, acc_block_x=best_blk[0], acc_block_y=best_blk[1])
            changed = True
        for (W, H) in sorted(sizes[c]):
            entries.append(dict(width=W, height=H, **cache[key]))
    merger.set_tuning([])
    if changed:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return entries
