"""Launch shapes of isa_ctx_set_tuning (the autotuner's knobs) change no
result: merges with other LK strip heights and accumulation blocks are bit
for bit those of the library's own choices; shapes out of range are refused;
the autotuner writes and reuses its JSON cache."""
import json

import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic, tune

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def burst(cuda):
    import torch
    b = synthetic.make_burst(640, 480, 4, seed=8, max_shift=4.0, max_rot_deg=0.2)
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    return b, raw


@pytest.mark.parametrize("scale", [1.5, 2.0])
def test_tuned_shapes_give_identical_merges(burst, scale):
    import torch
    b, raw = burst
    p = P.MergeParams()
    p.merge_scale = scale
    m = isa.Merger(b.width, b.height, b.n, p)
    info = isa.make_info(b)
    want = m.merge(raw, info).clone()
    for rows, bx, by in [(32, 64, 4), (96, 16, 16), (24, 128, 2)]:
        m.set_tuning([dict(width=b.width, height=b.height, lk_strip_rows=rows, acc_block_x=bx, acc_block_y=by)])
        got = m.merge(raw, info)
        torch.cuda.synchronize()
        assert torch.equal(got, want), (rows, bx, by)
    m.set_tuning([dict(width=0, height=0, lk_strip_rows=40)])  # the any-size entry
    assert torch.equal(m.merge(raw, info), want)
    m.close()


def test_bad_shapes_are_refused(burst):
    b, raw = burst
    m = isa.Merger(b.width, b.height, b.n, P.MergeParams())
    for e in [dict(acc_block_x=64, acc_block_y=8), dict(acc_block_x=24, acc_block_y=1), dict(lk_strip_rows=-1)]:
        with pytest.raises(isa.IsaError):
            m.set_tuning([e])
    m.close()


def test_autotuner_caches_its_choices(burst, tmp_path):
    import torch
    b, raw = burst
    p = P.MergeParams()
    p.merge_scale = 2.0
    m = isa.Merger(b.width, b.height, b.n, p)
    Wo, Ho = m.output_size(b.width, b.height)
    item = dict(raw=raw, info=isa.make_info(b), params=p, out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda"))
    path = tmp_path / "tuning.json"
    e1 = tune.tune(m, [item], cache_path=str(path), reps=1)
    cache = json.loads(path.read_text())
    assert len(cache) == 1 and len(e1) == 1 and e1[0]["width"] == b.width
    stamp = path.stat().st_mtime_ns
    e2 = tune.tune(m, [item], cache_path=str(path), reps=1)
    assert e2 == e1 and path.stat().st_mtime_ns == stamp  # from the cache, nothing rewritten
    m.close()
