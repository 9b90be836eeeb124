"""Merge parameters and tracking strategies.

`MergeParams` mirrors the `isa_params` struct of include/isa.h field by field.
Names and defaults are the DependencyProperty defaults of the reference
controller (PEFStudioDX/ImageStackAlignatorController.cs:443-675) and of
PatchTrackingLevel (PEFStudioDX/PatchTrackingLevel.cs:33-44); levels added
after the first use (2 * previous, 32, 4) as in AddPatchTrackingLevel
(ImageStackAlignatorController.cs:1572-1586).

The strategy helpers restate ShiftCollection's pair bookkeeping
(PEFStudioDX/ShiftCollection.cs:100-512): the number of pairs, the tracked
(reference, toTrack) pairs, the pair -> measurement index table and the
pair x one-to-one incidence matrix.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

FULL, ONLY_ON_REFERENCE, ON_REFERENCE_BLOCK, BLOCKS = 0, 1, 2, 3
SAMPLE_ROUND, SAMPLE_BILINEAR = 0, 1  # how the accumulation and the mask read a frame at the flow
MAX_LEVELS = 8


@dataclass
class TrackingLevel:
    """PatchTrackingLevel (PatchTrackingLevel.cs:27-63)."""
    resize_level: int = 1
    tile_size: int = 32
    max_shift: int = 2


def default_levels(count: int = 4) -> List[TrackingLevel]:
    levels = [TrackingLevel()]
    while len(levels) < count:
        levels.append(TrackingLevel(levels[-1].resize_level * 2, 32, 4))
    return levels


@dataclass
class MergeParams:
    sigma_debayer_tracking: float = 0.5
    sigma_debayer_accumulation: float = 0.5
    high_pass: float = 0.01
    high_pass_sigma: float = 0.0025
    clear_axis: int = 0
    matching_threshold: float = 1.0
    sigma_structure_tensor: float = 1.0
    dth: float = 0.001
    dtr: float = 0.006
    k_detail: float = 0.25
    k_denoise: float = 3.0
    k_stretch: float = 4.0
    k_shrink: float = 2.0
    iterations_lk: int = 3
    window_size_lk: int = 11
    erode_size: int = 5
    min_det_lk: float = 0.01
    threshold_m: float = 100000.0
    tracking_strategy: int = FULL
    tracking_block_size: int = 5
    green_channel_only: bool = False
    levels: List[TrackingLevel] = field(default_factory=default_levels)
    # extensions (reference-equivalent defaults)
    super_resolution: bool = False   # reference SuperResolution: central crop at 2x
    merge_scale: float = 0.0         # 0: reference mode (1x plain, or 2x crop when super_resolution)
    robust_s: float = 1.5            # RobustnessModell.cu:472 literal
    robust_t: float = 0.12           # RobustnessModell.cu:476 literal
    sample_mode: int = SAMPLE_ROUND  # SAMPLE_BILINEAR: blend of the four integer shifts, continuous in the flow

    def f32(self, name):
        return float(np.float32(getattr(self, name)))


def shift_count(n: int, strategy: int, block: int) -> int:
    """ShiftCollection.GetShiftCount (ShiftCollection.cs:100-121)."""
    if strategy == FULL:
        return int((n - 1) * (np.float32(n) / np.float32(2.0)))
    if strategy == ONLY_ON_REFERENCE:
        return n - 1
    if strategy == ON_REFERENCE_BLOCK:
        return int((block - 1) * (np.float32(block) / np.float32(2.0))) + block * (n - block)
    if strategy == BLOCKS:
        return int(-0.5 * block * (block - 2 * n + 1))
    return 0


def effective_block(n: int, block: int) -> int:
    """ShiftCollection constructor clamp (ShiftCollection.cs:495-502)."""
    return n - 1 if block >= n else block


def _ref_block_bounds(n, ref, block):
    if ref < n // 2:
        first = max(ref - block // 2, 0)
        last = first + block - 1
    else:
        last = min(ref + block // 2, n - 1)
        first = last - block + 1
    return first, last


def shift_pairs(n: int, ref: int, strategy: int, block: int) -> List[Tuple[int, int]]:
    """FillShiftPairs (ShiftCollection.cs:275-377): tracking order."""
    block = effective_block(n, block)
    pairs = []
    if strategy == FULL:
        for r in range(n):
            for t in range(r + 1, n):
                pairs.append((r, t))
    elif strategy == ONLY_ON_REFERENCE:
        for t in range(n):
            if t != ref:
                pairs.append((ref, t))
    elif strategy == ON_REFERENCE_BLOCK:
        first, last = _ref_block_bounds(n, ref, block)
        for s in range(block - 1):
            count = block - 1 - s
            for line in range(count):
                pairs.append((line + first, line + first + block - count))
        for i in range(first):
            for tb in range(first, last + 1):
                pairs.append((tb, i))
        for i in range(last + 1, n):
            for tb in range(first, last + 1):
                pairs.append((tb, i))
    elif strategy == BLOCKS:
        for s in range(block):
            count = (n - 1) - s
            for line in range(count):
                pairs.append((line, line + n - count))
    return pairs


def index_table(n: int, ref: int, strategy: int, block: int) -> np.ndarray:
    """FillIndexTable (ShiftCollection.cs:379-488): [from, to] -> measurement row."""
    block = effective_block(n, block)
    idx = -np.ones((n, n), dtype=np.int64)
    c = 0
    if strategy == FULL:
        for d in range(1, n):
            for f in range(n - d):
                idx[f, f + d] = c; c += 1
    elif strategy == ONLY_ON_REFERENCE:
        for t in range(n):
            if t != ref:
                idx[ref, t] = c; c += 1
    elif strategy == ON_REFERENCE_BLOCK:
        first, last = _ref_block_bounds(n, ref, block)
        for s in range(block - 1):
            count = block - 1 - s
            for line in range(count):
                idx[line + first, line + first + block - count] = c; c += 1
        for i in range(first):
            for tb in range(first, last + 1):
                idx[tb, i] = c; c += 1
        for i in range(last + 1, n):
            for tb in range(first, last + 1):
                idx[tb, i] = c; c += 1
    elif strategy == BLOCKS:
        for d in range(1, block + 1):
            for f in range(n - d):
                idx[f, f + d] = c; c += 1
    return idx


def shift_matrix(n: int, ref: int, strategy: int, block: int) -> np.ndarray:
    """CreateShiftMatrix (ShiftCollection.cs:123-273) as an m x (n-1) row-major
    array: row = measurement (pair), column = one-to-one shift i -> i+1."""
    block = effective_block(n, block)
    m = shift_count(n, strategy, block)
    A = np.zeros((m, n - 1), dtype=np.float64)
    if strategy == FULL:
        c = 0
        for s in range(n - 1):
            count = (n - 1) - s
            for line in range(count):
                A[c, line:line + (n - 1) - count + 1] = 1
                c += 1
    elif strategy == ONLY_ON_REFERENCE:
        for img in range(n - 1):
            if img < ref:
                A[img, img:ref] = -1
            else:
                A[img, ref:img + 1] = 1
    elif strategy == ON_REFERENCE_BLOCK:
        first, last = _ref_block_bounds(n, ref, block)
        c = 0
        for s in range(block - 1):
            count = block - 1 - s
            for line in range(count):
                A[c, line + first:line + first + block - count] = 1
                c += 1
        for i in range(first):
            for tb in range(first, last + 1):
                A[c, i:tb] = -1
                c += 1
        for i in range(last + 1, n):
            for tb in range(first, last + 1):
                A[c, tb:i] = 1
                c += 1
    elif strategy == BLOCKS:
        c = 0
        for s in range(block):
            count = (n - 1) - s
            for line in range(count):
                A[c, line:line + (n - 1) - count + 1] = 1
                c += 1
    return A
