"""Golden vectors of the FP32 GammasRGB (Kernels/kernel.cu:290-332) from the
reference's own kernel body compiled for the host in float
(oracle/_ref/libref32.so), for tests/test_oracle_post.py: they pin the
post-processing restatement's gamma step (oracle/post.py) without the
reference sources present.

    make -C oracle && python tests/golden/make_post_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pipeline as PL  # noqa: E402


def gamma_inputs():
    rng = np.random.default_rng(2024)
    v = (rng.random((48, 64, 3)) * 1.3 - 0.1).astype(np.float32)
    edge = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 1.0, 0.0031308, 0.0031309, 1e-30, 0.9999999, 1.0000001, 0.5], np.float32)
    v.reshape(-1)[:edge.size] = edge
    return v


def main():
    lib = PL.StageLib("ref32")
    v = gamma_inputs()
    np.savez_compressed(os.path.join(HERE, "post_golden.npz"), in_gamma32=v, out_gamma32=lib.gamma_srgb(v))
    print("wrote post_golden.npz")


if __name__ == "__main__":
    main()
