"""The small CPU-runnable burst at its real size, GPU against the FP64 oracle.

2048 x 1536 RGGB, 14-bit (black 512, white 16383), 8 frames with shifts of
up to 6 px and rotations of up to 0.2 degrees, Poisson-Gaussian noise
(a = 4e-4, b = 2e-6); the reference's plain merge (scale 1, ApplyWeighting
threshold 1), 4-level pyramid (1, 32, 2), (2, 32, 4), (4, 32, 4), (8, 32, 4),
Full strategy (28 pairs), 3 LK iterations. Tile stride is the tile size, as
in the reference (kernel.cu:220).

Checked through the C ABI (isa_merge_burst):
- the integer tile shift (first minimum of the L2 map, kernel.cu:422-546)
  of every tile of every pair at every level, bit-exact wherever the search
  block sits at the same integer offset, except ties (best and second-best
  L2 within a relative 1e-5), which are counted;
- the merged FP32 RGB: max |GPU - FP64| <= 1e-4 of the white level over every
  pixel whose discrete decisions (round(s * flow), round(flow / 2) through
  the eroded mask, w < threshold) match the oracle's; the pixels that read a
  differing decision are identified, counted and bounded (oracle/parity.py);
- the one-to-one shifts of the finest level and the dense flows."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

import parity
import pipeline as PL

pytestmark = pytest.mark.gpu

W, H, N = 2048, 1536, 8


@pytest.fixture(scope="module")
def case(oracle):
    burst = synthetic.make_burst(W, H, N, seed=0, max_shift=6.0, max_rot_deg=0.2, noise_a=4e-4, noise_b=2e-6)
    p = P.MergeParams()
    p.levels = P.default_levels(4)
    keep = {}
    want = PL.merge_burst(burst, p, lib=oracle, keep=keep)
    return burst, p, keep, want


def test_config0_matches_oracle(cuda, case):
    import torch
    burst, p, keep, want = case
    pairs, _ = isa.tracking_pairs(N, 0, p.tracking_strategy, p.tracking_block_size)
    assert len(pairs) == 28
    m = isa.Merger(W, H, N, p)
    rec = torch.zeros(isa.track_record_ints(m.params, W, H, len(pairs)), dtype=torch.int32, device="cuda")
    m.set_track_record(rec)
    raw = torch.from_numpy(np.ascontiguousarray(burst.raw).view(np.int16)).cuda()
    out = m.merge(raw, isa.make_info(burst))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    # integer tile shifts, every pair at every level
    ts = parity.track_parity(rec.cpu().numpy(), keep, [tuple(map(int, rt)) for rt in pairs], p.levels, W, H)
    print("tile shifts:", ts)
    assert ts["argmin_checked"] >= 0.99 * ts["tiles"]
    # one-to-one shifts of the finest level
    xs, tx, ty = m.debug_shifts()
    x = isa.device_copy(xs, (ty * tx, N - 1, 2), torch.float32).cpu().numpy()
    dx = np.abs(x - keep["x"]).max(axis=(1, 2))
    assert np.percentile(dx, 99) < 1e-3, np.percentile(dx, 99)
    # dense flows
    flows, masks = m.flows_masks(N, W, H)
    for i in range(1, N):
        df = np.abs(flows[i] - keep["flow"][i]).max(axis=2)
        assert np.percentile(df, 99.9) < 1e-3, (i, np.percentile(df, 99.9))
    # merged image over decision-matched pixels
    geom = PL.out_geometry(W, H, p)
    sub = PL.merge_tail(burst, p, flows, masks, m.kernel_params(W, H), PL.StageLib("oracle64"))
    st = parity.merge_parity(got, want.image, flows, keep["flow"], masks, keep["mask"], geom, p.erode_size, wsum_orc=want.wsum,
                             wsum_gpu=m.weight_sums(W, H), want_sub=sub.image, wsum_sub=sub.wsum, max_excluded=0.01)
    print("merged image:", st)
    m.set_track_record(None)
    m.close()
