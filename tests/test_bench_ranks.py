"""Rank logic of bench.py with world size 2 over gloo on CPU: every rank
merges its own burst (distinct seeds), the reported step time is the max
over ranks, the job value counts every rank's output, and the reference arm
runs on rank 0 only. No GPU and no merge is involved."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        got = bench.reduce_max(ms, dist, "cpu")
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.burst_seed(rank))
        buf = io.StringIO()

        class A:
            steps, warmup, gpus = 1, 0, world
        if rank != 0:  # rank 0 would run the host reference; only its skip path is exercised here
            with redirect_stdout(buf):
                rc = bench.run_reference(A)
        else:
            rc = 0
        out[rank] = dict(max_ms=got, seeds=seeds, rc=rc, printed=buf.getvalue(), value=bench.job_value(world, 96.256, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        assert res[r]["max_ms"] == 150.0
        assert res[r]["seeds"] == [1000, 1001]
        assert res[r]["value"] == pytest.approx(2 * 96.256 / 0.150)
    assert res[1]["rc"] == 0 and res[1]["printed"] == ""


def test_single_rank_value_and_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(12.5, None, "cpu") == 12.5
    assert bench.job_value(1, 96.256, 200.0) == pytest.approx(481.28)
    json.dumps({"v": bench.job_value(1, 1.0, 1.0)})
