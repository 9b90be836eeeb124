"""Burst assignment of isa_merge_batch (isa_batch_plan, host only) over
contexts on several devices, and the rank split built on it (isa.rank_bursts)
over a gloo process group of world size 2."""
import os

import numpy as np
import pytest

from imagestackalignator_b200 import isa


def plan_restated(work, bdev, cdev):
    load = [0.0] * len(cdev)
    out = []
    for w, d in zip(work, bdev):
        cand = [k for k in range(len(cdev)) if d < 0 or cdev[k] == d]
        if not cand:
            out.append(-1)
            continue
        k = min(cand, key=lambda i: (load[i], i))
        load[k] += w
        out.append(k)
    return out


def test_bursts_stay_on_their_device():
    cdev = [0, 0, 1, 1]
    work = [5.0, 3.0, 4.0, 1.0, 2.0, 2.0]
    bdev = [0, 0, 1, 1, 0, -1]
    a = isa.batch_plan(work, bdev, cdev)
    assert a == [0, 1, 2, 3, 1, 3]
    for b, k in enumerate(a):
        assert bdev[b] < 0 or cdev[k] == bdev[b]


def test_no_context_on_a_device():
    a = isa.batch_plan([1.0, 1.0], [0, 2], [0, 1])
    assert a == [0, -1]


def test_plan_matches_the_restated_rule():
    rng = np.random.default_rng(0)
    for _ in range(50):
        nctx, nb = int(rng.integers(1, 6)), int(rng.integers(0, 40))
        cdev = [int(v) for v in rng.integers(0, 3, nctx)]
        bdev = [int(v) for v in rng.integers(-1, 3, nb)]
        work = [float(v) for v in rng.uniform(1, 100, nb)]
        assert isa.batch_plan(work, bdev, cdev) == plan_restated(work, bdev, cdev)


def test_rank_split_is_a_partition_balanced_by_work():
    rng = np.random.default_rng(1)
    work = [float(v) for v in rng.integers(2, 12, 64) * rng.integers(4, 31, 64)]  # MP x frames, config-3 style
    parts = isa.rank_bursts(work, 8)
    got = sorted(b for p in parts for b in p)
    assert got == list(range(64))
    loads = [sum(work[b] for b in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)


def _rank_main(rank, world, port, work, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    mine = isa.rank_bursts(work, world)[rank]
    # stand-in for each rank's merges: a checksum per burst it owns
    done = torch.zeros(len(work), dtype=torch.float64)
    for b in mine:
        done[b] = 1000.0 * b + work[b]
    dist.all_reduce(done)
    q.put((rank, mine, done.tolist()))
    dist.destroy_process_group()


def test_two_ranks_over_gloo_merge_every_burst_once():
    import multiprocessing as mp
    import socket
    rng = np.random.default_rng(2)
    work = [float(v) for v in rng.uniform(1, 50, 23)]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, work, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert sorted(res[0][1] + res[1][1]) == list(range(len(work)))
    want = [1000.0 * b + w for b, w in enumerate(work)]
    for _, _, done in res:
        assert np.allclose(done, want)
