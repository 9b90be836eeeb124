import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libisa.so")


def _ensure_oracle_built():
    lib = os.path.join(ROOT, "oracle", "_build", "liboracle64.so")
    if not os.path.exists(lib):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle_built()
    import pipeline as PL
    return PL.StageLib("oracle64")


@pytest.fixture(scope="session")
def small_burst():
    from imagestackalignator_b200 import synthetic
    return synthetic.make_burst(512, 384, 4, seed=7, max_shift=6, max_rot_deg=0.2)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    from imagestackalignator_b200 import isa
    isa.lib()
    return torch.device("cuda")
