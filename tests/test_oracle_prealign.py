"""The restated global pre-alignment (oracle/pipeline.py: ScanAngles and
PreAlignmentStore) on CPU: a burst with known translations and rotations
(the reference's test mode synthesises the same kind of burst,
TestRawFile.cs:39-64) is recovered to a pixel and to about two fine angle
steps (the correlation peak is a coarse angle estimator), and the store
picks the reference that minimises the remaining shift."""
import numpy as np
import pytest

import pipeline as PL
from imagestackalignator_b200 import params as P, synthetic


@pytest.fixture(scope="module")
def scene_burst():
    return synthetic.make_burst(384, 288, 3, seed=5, max_shift=6.0, max_rot_deg=0.5)


def test_scan_recovers_translation_and_rotation(oracle, scene_burst):
    b = scene_burst
    p = P.MergeParams()
    imgs = np.stack([PL.bw_image(oracle, b, i, p.sigma_debayer_tracking, True, p) for i in range(b.n)])
    init, (shifts, rots, ref) = PL.prealign_images(imgs)
    for i in range(1, b.n):
        x, y, ang, val = init[i]
        assert abs(x - b.shifts[i, 0]) <= 1.0 and abs(y - b.shifts[i, 1]) <= 1.0, (i, init[i], b.shifts[i])
        assert abs(ang + b.rotations[i]) <= 0.2, (i, ang, b.rotations[i])  # about two fine steps
    assert 0 <= ref < b.n - 1


def test_store_matches_hand_computed_case():
    init = [(0, 0, 0, 0), (4.0, -2.0, 0.2, 1), (10.0, -1.0, 0.1, 1), (12.0, 3.0, -0.1, 1)]
    shifts, rots, ref = PL.prealign_store(init)
    # remaining total shift per candidate reference i: -sum(basic[:i]) + sum(basic[i:]) -> frame 1 is the middle
    basic = np.diff(np.array(init, float)[:, :3], axis=0)
    tot = [np.hypot(*(-basic[:i, :2].sum(0) + basic[i:, :2].sum(0))) for i in range(3)]
    assert ref == int(np.argmin(tot))
    np.testing.assert_allclose(shifts[ref], 0, atol=0)
    np.testing.assert_allclose(shifts[:, 0] - shifts[0, 0], np.array(init)[:, 0], atol=1e-6)
    np.testing.assert_allclose(rots - rots[0], np.array(init)[:, 2], atol=1e-6)


def test_rotation_by_zero_is_identity():
    rng = np.random.default_rng(1)
    img = rng.uniform(0, 1, (20, 30))
    np.testing.assert_allclose(PL.rotate_cubic(img, 0.0), img, atol=1e-12)


def test_cross_correlation_product_is_the_reference_kernel():
    """The scan's cross-correlation product conj(R) * T (oracle scan_angles, and
    the fused multiply of the GPU's column transforms that test_gpu_prealign
    checks against it) is the reference's own conjugateComplexMulKernel
    (kernel.cu:395-411), which PreAlignment.cs:200 calls with the reference
    spectrum as its first, conjugated operand; run through its host build."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref64.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built here (no reference checkout)")
    lib = ctypes.CDLL(path)
    rng = np.random.default_rng(3)
    n = 4099
    R = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    T = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a = np.ascontiguousarray(np.stack([R.real, R.imag], -1))
    b = np.ascontiguousarray(np.stack([T.real, T.imag], -1))
    lib.ref_conj_mul(a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(n))
    got = b[:, 0] + 1j * b[:, 1]
    # numpy's complex product rounds differently from the kernel's four scalar products (an ulp): the convention
    # (which spectrum is conjugated) is what is pinned; the other one is far off
    np.testing.assert_allclose(got, np.conj(R) * T, rtol=1e-12, atol=0)
    assert np.abs(got - np.conj(T) * R).max() > 1.0
