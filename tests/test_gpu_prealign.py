"""Global pre-alignment on the GPU (isa_prealign_burst) against the restated
ScanAngles / PreAlignmentStore of oracle/pipeline.py, run on the GPU's own
tracking images (isa_bw_image), so that the comparison isolates the scan:
the rotation, the FFT cross-correlation and the arg-max. Integer shifts and
the chosen angles must agree exactly; the correlation values to FP32
precision."""
import ctypes

import numpy as np
import pytest

import pipeline as PL
from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def burst():
    return synthetic.make_burst(512, 384, 4, seed=9, max_shift=8.0, max_rot_deg=0.5)


def test_prealign_matches_oracle_scan(cuda, burst):
    import torch
    b = burst
    p = P.MergeParams()
    m = isa.Merger(b.width, b.height, b.n, p)
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    shifts, rots, ref, scan = m.prealign(raw, info)
    # the same tracking images through the operator entry point
    imgs = []
    for i in range(b.n):
        out = torch.empty((b.height, b.width), dtype=torch.float32, device="cuda")
        isa.check(isa.lib().isa_bw_image(m.ctx, isa.vp(raw[i]), ctypes.c_size_t(b.width * 2), b.width, b.height, ctypes.byref(info),
                                         ctypes.c_float(p.sigma_debayer_tracking), 1, isa.vp(out), ctypes.c_size_t(b.width * 4), None))
        imgs.append(out)
    torch.cuda.synchronize()
    imgs = np.stack([t.cpu().numpy().astype(np.float64) for t in imgs])
    init, (w_shifts, w_rots, w_ref) = PL.prealign_images(imgs)
    for i in range(1, b.n):
        assert tuple(scan[i, :3]) == pytest.approx(init[i][:3], abs=1e-9), (i, scan[i], init[i])
        assert scan[i, 3] == pytest.approx(init[i][3], rel=1e-4)
        # and the scan finds the synthetic motion: translation to a pixel, rotation to the fine step
        assert abs(scan[i, 0] - b.shifts[i, 0]) <= 1.0 and abs(scan[i, 1] - b.shifts[i, 1]) <= 1.0
        assert abs(scan[i, 2] + b.rotations[i]) <= 0.2  # the correlation peak resolves the angle to about two fine steps
    assert ref == w_ref
    np.testing.assert_array_equal(shifts, w_shifts)
    np.testing.assert_allclose(rots, w_rots, atol=1e-6)
    # the result feeds the merge directly
    out = m.merge(raw, info, shifts=shifts, rotations=rots, reference=ref)
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    m.close()


def test_prealign_rejects_bad_arguments(cuda, burst):
    import torch
    b = burst
    m = isa.Merger(b.width, b.height, b.n, P.MergeParams())
    info = isa.make_info(b)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    with pytest.raises(isa.IsaError):
        m.prealign(raw, info, increment=0.0)
    with pytest.raises(isa.IsaError):
        m.prealign(raw, info, increment=1e-4, range_deg=10.0)  # too many angles per scan
    m.close()
