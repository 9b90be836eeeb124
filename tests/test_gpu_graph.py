"""A batch of uneven bursts captured as a CUDA graph (isa_batch_graph_create)
and replayed (isa_batch_graph_launch): every replay gives the outputs of the
same batch merged directly (isa_merge_batch), bit for bit, also after the
contexts merged other bursts between replays."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

pytestmark = pytest.mark.gpu

SPECS = [(512, 384, 4, 2.0, "RGGB"), (640, 480, 3, 1.0, "BGGR"), (448, 352, 5, 2.0, "GRBG"), (448, 320, 4, 1.5, "RGGB")]


@pytest.fixture(scope="module")
def batch(cuda):
    import torch
    items = []
    for k, (W, H, n, s, cfa) in enumerate(SPECS):
        b = synthetic.make_burst(W, H, n, seed=40 + k, max_shift=4.0, max_rot_deg=0.2, cfa=cfa)
        q = P.MergeParams()
        q.merge_scale = s
        Wo, Ho = isa.output_size(isa.make_params(q), W, H)
        items.append(dict(raw=torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda(), info=isa.make_info(b), params=q,
                          out=torch.empty((Ho, Wo, 3), dtype=torch.float32, device="cuda")))
    p = P.MergeParams()
    p.merge_scale = 2.0
    mergers = [isa.Merger(640, 480, 5, p) for _ in range(2)]
    return items, mergers


def test_graph_replays_equal_the_direct_batch(batch):
    import torch
    items, mergers = batch
    streams = [torch.cuda.Stream() for _ in mergers]
    origin = torch.cuda.Stream()
    st = isa.merge_batch(mergers, items, streams)
    assert not any(st), st
    torch.cuda.synchronize()
    want = [it["out"].clone() for it in items]
    for it in items:
        it["out"].zero_()
    g = isa.BatchGraph(mergers, items, streams, origin)
    torch.cuda.synchronize()
    assert all(float(it["out"].abs().sum()) == 0.0 for it in items)  # capturing runs nothing
    for rep in range(2):
        for it in items:
            it["out"].zero_()
        torch.cuda.synchronize()
        g.launch(origin)
        origin.synchronize()
        for k, it in enumerate(items):
            assert torch.equal(it["out"], want[k]), (rep, k)
        # other work on the contexts between replays: a different burst on each
        other = synthetic.make_burst(600, 400, 5, seed=99, max_shift=3.0)
        o = dict(raw=torch.from_numpy(np.ascontiguousarray(other.raw).view(np.int16)).cuda(), info=isa.make_info(other),
                 out=torch.empty(mergers[0].output_size(600, 400)[::-1] + (3,), dtype=torch.float32, device="cuda"))
        for m in mergers:
            m.merge(o["raw"], o["info"], o["out"])
        torch.cuda.synchronize()
    g.close()


def test_merges_after_a_capture_use_their_own_tables(batch):
    """The capture runs the host side of the merges but none of their copies:
    a direct merge right after it, of the size captured last, must still
    upload its own transform tables (the context held another size before)."""
    import torch
    items, mergers = batch
    m0 = mergers[0]
    s0, origin = torch.cuda.Stream(), torch.cuda.Stream()
    want = []
    for it in items:
        one = dict(it, out=torch.empty_like(it["out"]))
        assert not any(isa.merge_batch([m0], [one]))
        want.append(one["out"])
    other = synthetic.make_burst(600, 400, 5, seed=98, max_shift=3.0)
    o_out = torch.empty(m0.output_size(600, 400)[::-1] + (3,), dtype=torch.float32, device="cuda")
    m0.merge(torch.from_numpy(np.ascontiguousarray(other.raw).view(np.int16)).cuda(), isa.make_info(other), o_out)
    g = isa.BatchGraph([m0], items, [s0], origin)
    last = dict(items[-1], out=torch.empty_like(items[-1]["out"]))
    assert not any(isa.merge_batch([m0], [last]))
    torch.cuda.synchronize()
    assert torch.equal(last["out"], want[-1])
    g.close()


def test_graph_arguments_are_checked(batch):
    import torch
    items, mergers = batch
    s = torch.cuda.Stream()
    with pytest.raises(isa.IsaError):
        isa.BatchGraph(mergers, items, [s, s], torch.cuda.Stream())  # the same stream twice
    with pytest.raises(isa.IsaError):
        isa.BatchGraph(mergers[:1], items, [s], s)  # the origin among the streams
