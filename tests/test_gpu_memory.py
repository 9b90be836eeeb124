"""Calls on a context allocate nothing: merges of bursts of three different
frame sizes (the full-frame transforms re-plan for each size from tables in
the context), the batch entry point over them, and the adjoint all leave
the device's free memory unchanged once the context exists."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu


def test_calls_allocate_nothing(cuda):
    import torch
    p = P.MergeParams()
    p.merge_scale = 2.0
    sizes = [(640, 480, 4), (512, 384, 3), (768, 512, 5)]  # every level of the default 4-level pyramid has tiles
    bursts = [synthetic.make_burst(w, h, n, seed=w + n, max_shift=3, max_rot_deg=0.1) for w, h, n in sizes]
    m = isa.Merger(768, 512, 5, p)
    raws = [torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda() for b in bursts]
    infos = [isa.make_info(b) for b in bursts]
    outs = [torch.empty((h * 2, w * 2, 3), dtype=torch.float32, device="cuda") for w, h, _ in sizes]
    targets = [torch.rand_like(o) for o in outs]
    items = [dict(raw=r, info=i, out=o) for r, i, o in zip(raws, infos, outs)]
    # one round of everything first (loads the library's device code, fills torch's caches)
    for r, i, o, t in zip(raws, infos, outs, targets):
        m.merge(r, i, o)
        m.backward(r, i, t)
    isa.merge_batch([m], items)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        for r, i, o, t in zip(raws, infos, outs, targets):
            m.merge(r, i, o)
            m.backward(r, i, t)
        st = isa.merge_batch([m], items)
        assert not any(st), st
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    m.close()


def test_flow_adjoint_and_parameter_changes_allocate_nothing(cuda):
    """isa_merge_backward_tiles (sample mode BILINEAR, scratch from the context),
    isa_ctx_set_params and isa_ctx_set_tuning between calls, over three sizes."""
    import torch
    p = P.MergeParams()
    p.merge_scale = 1.5
    p.sample_mode = P.SAMPLE_BILINEAR
    sizes = [(640, 480, 4), (512, 384, 3), (768, 512, 5)]
    bursts = [synthetic.make_burst(w, h, n, seed=2 * w + n, max_shift=3, max_rot_deg=0.1) for w, h, n in sizes]
    m = isa.Merger(768, 512, 5, p)
    raws = [torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda() for b in bursts]
    infos = [isa.make_info(b) for b in bursts]
    targets = [torch.rand((*m.output_size(w, h)[::-1], 3), device="cuda") for w, h, _ in sizes]
    q = P.MergeParams(**vars(p))
    q.k_detail = 0.3

    def round_of_calls():
        for k, (r, i, t) in enumerate(zip(raws, infos, targets)):
            m.set_params(q if k % 2 else p)
            m.set_tuning([dict(width=sizes[k][0], height=sizes[k][1], lk_strip_rows=32 + 16 * k)])
            m.backward_tiles(r, i, t)

    round_of_calls()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        round_of_calls()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    m.close()
