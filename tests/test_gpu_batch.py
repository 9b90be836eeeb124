"""Batched merge of several bursts (isa_merge_batch) over several contexts and
streams: every output must equal, bit for bit, the output of merging that
burst alone with isa_merge_burst and the same parameters (the kernels and
their reduction orders do not depend on which context or stream runs them)."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu


def to_dev(raw):
    import torch
    return torch.from_numpy(np.ascontiguousarray(raw).view(np.int16)).cuda()


def _bursts():
    specs = [(640, 480, 5, "RGGB", 0.0), (512, 384, 4, "GRBG", 0.0), (640, 448, 3, "BGGR", 1.5), (384, 320, 6, "GBRG", 2.0),
             (576, 416, 2, "RGGB", 0.0)]
    out = []
    for i, (w, h, n, cfa, scale) in enumerate(specs):
        b = synthetic.make_burst(w, h, n, seed=40 + i, max_shift=5, max_rot_deg=0.1, cfa=cfa)
        out.append((b, scale))
    return out


def test_batch_equals_single_merges(cuda):
    import torch
    bursts = _bursts()
    W = max(b.width for b, _ in bursts)
    H = max(b.height for b, _ in bursts)
    N = max(b.n for b, _ in bursts)
    base = P.MergeParams()
    base.merge_scale = 2.0          # the contexts size their outputs for the largest scale used
    singles = []
    for b, scale in bursts:
        p = P.MergeParams()
        p.merge_scale = scale
        out = isa.Merger(b.width, b.height, b.n, p).merge(to_dev(b.raw), isa.make_info(b))
        torch.cuda.synchronize()
        singles.append(out.cpu().numpy())
    mergers = [isa.Merger(W, H, N, base) for _ in range(3)]
    streams = [torch.cuda.Stream() for _ in mergers]
    items, raws = [], []
    for b, scale in bursts:
        p = P.MergeParams()
        p.merge_scale = scale
        raw = to_dev(b.raw)
        raws.append(raw)
        Wo, Ho = isa.output_size(isa.make_params(p), b.width, b.height)
        out = torch.full((Ho, Wo, 3), float("nan"), dtype=torch.float32, device="cuda")
        items.append(dict(raw=raw, info=isa.make_info(b), out=out, params=p))
    torch.cuda.synchronize()
    status = isa.merge_batch(mergers, items, streams)
    torch.cuda.synchronize()
    assert status == [0] * len(items)
    for it, want in zip(items, singles):
        got = it["out"].cpu().numpy()
        assert got.shape == want.shape
        assert np.array_equal(got, want)
    # a second batch reusing the contexts gives the same images again
    for it in items:
        it["out"].fill_(float("nan"))
    status = isa.merge_batch(mergers, items, streams)
    torch.cuda.synchronize()
    assert status == [0] * len(items)
    for it, want in zip(items, singles):
        assert np.array_equal(it["out"].cpu().numpy(), want)


def test_batch_reports_bad_bursts(cuda):
    import torch
    b = synthetic.make_burst(384, 320, 3, seed=7, max_shift=4, max_rot_deg=0.0)
    m = isa.Merger(384, 320, 3, P.MergeParams())
    raw = to_dev(b.raw)
    Wo, Ho = m.output_size(384, 320)
    good = dict(raw=raw, info=isa.make_info(b), out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda"))
    p = P.MergeParams()
    p.levels = p.levels[:2]
    bad = dict(raw=raw, info=isa.make_info(b), out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda"), params=p)
    status = isa.merge_batch([m], [good, bad, good])
    torch.cuda.synchronize()
    assert status[0] == 0 and status[2] == 0
    assert status[1] == isa.ISA_EINVAL
    assert np.isfinite(good["out"].cpu().numpy()).all()
