"""Generate the golden vectors of tests/golden/golden.npz from the reference's
own kernel bodies (oracle/_ref/libref64.so: Kernels/*.cu compiled for the
host with float -> double).

The reference ships no tests, fixtures or known-answer vectors, so these
vectors are the reference itself run on small seeded inputs; the committed
file lets the CPU tests pin the FP64 restatement (oracle/isa_oracle.c)
without the reference sources present.

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import golden_cases  # noqa: E402
import pipeline as PL  # noqa: E402


def main():
    lib = PL.StageLib("ref64")
    out = golden_cases.run_all(lib)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
