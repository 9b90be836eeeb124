"""The data-parallel parameter fit (imagestackalignator_b200.fit.adam_fit with
a process group): each rank's loss and eight gradients are summed with one
all-reduce per step, so two gloo ranks with different data take identical
steps, equal to one process fitting the summed loss. The per-rank losses are
stand-ins with known gradients (the GPU adjoint is checked in
test_gpu_adjoint*.py); the fit's own log-space Adam is checked to converge."""
import os

import numpy as np

from imagestackalignator_b200 import fit

THETA0 = np.array([0.25, 3.0, 0.001, 0.006, 4.0, 2.0, 1.5, 0.12])


def rank_loss(r):
    rng = np.random.default_rng(10 + r)
    c = np.log(THETA0) + rng.normal(0, 0.5, 8)
    w = rng.uniform(0.5, 2.0, 8)

    def fn(theta):
        d = np.log(theta) - c
        return float(np.sum(w * d * d)), 2 * w * d / theta

    return fn, c, w


def test_single_process_fit_converges():
    fn0, c0, w0 = rank_loss(0)
    theta, losses = fit.adam_fit(fn0, THETA0, 600, lr=0.02)
    assert losses[-1] < 1e-3 * losses[0]
    np.testing.assert_allclose(np.log(theta), c0, atol=2e-2)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fn, _, _ = rank_loss(rank)
    theta, losses = fit.adam_fit(fn, THETA0, 200, group=dist.group.WORLD)
    q.put((rank, theta.tolist(), losses))
    dist.destroy_process_group()


def test_two_ranks_take_the_steps_of_the_summed_loss():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, t0, l0), (_, t1, l1) = res
    assert t0 == t1 and l0 == l1  # every rank holds the same parameters
    fa, _, _ = rank_loss(0)
    fb, _, _ = rank_loss(1)

    def both(theta):
        la, ga = fa(theta)
        lb, gb = fb(theta)
        return la + lb, ga + gb

    theta, losses = fit.adam_fit(both, THETA0, 200)
    np.testing.assert_allclose(t0, theta, rtol=1e-12)
    np.testing.assert_allclose(l0, losses, rtol=1e-12)
