"""The multi-GPU plumbing on CPU: view partitioning, and the one gradient all_reduce over two gloo
ranks (the same calls run over NCCL on GPUs)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from aniso_b200 import multigpu, scenes


def test_partition_covers_every_view_once_and_balances():
    cams = scenes.fibonacci_cameras(64, 10.0, scenes.RESOLUTIONS_4, seed=3)
    costs = [multigpu.view_cost(c.width, c.height, 1_000_000) for c in cams]
    for world in (1, 2, 4, 8):
        shares = multigpu.partition_views(costs, world)
        flat = sorted(k for s in shares for k in s)
        assert flat == list(range(64))
        loads = [sum(costs[k] for k in s) for s in shares]
        assert max(loads) - min(loads) <= max(costs)  # greedy LPT bound
        assert shares == multigpu.partition_views(costs, world)  # deterministic


def test_partition_more_ranks_than_views():
    shares = multigpu.partition_views([5, 3], 4)
    assert shares == [[0], [1], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cams = scenes.ring_cameras(16, 8.0, 1280, 720, 1100.0)
        mine = multigpu.my_views(cams, 740_000, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # per-rank gradients of two parameter tensors; after the exchange every rank has the sum
        g1 = torch.full((5, 3), float(rank + 1))
        g2 = torch.arange(4, dtype=torch.float32) * (rank + 1)
        multigpu.allreduce_gradients([g1, None, g2])
        q.put((rank, gathered, g1.tolist(), g2.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_and_gradient_allreduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, g1, g2 in out:
        assert sorted(k for s in gathered for k in s) == list(range(16))
        assert g1 == [[3.0] * 3] * 5
        assert g2 == [0.0, 3.0, 6.0, 9.0]


def _grad_worker(rank, world, port, q):
    """Each rank differentiates its share of the views (the FP64 adjoint of the renderer, on the
    CPU) and the shares are summed with the one all_reduce a multi-GPU training step makes."""
    import numpy as np

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, cams, targets = _grad_case()
        R = oracle.Restatement()
        mine = multigpu.my_views(cams, params[0].shape[0], rank, world)
        acc = [torch.zeros(p.shape, dtype=torch.float64) for p in params]
        for k in mine:
            img = R.train_forward_f64(params, cams[k])
            for a, g in zip(acc, R.train_backward_f64(params, cams[k], 2 * (img - targets[k]))):
                a += torch.from_numpy(g)
        multigpu.allreduce_gradients(acc)
        q.put((rank, mine, [a.numpy() for a in acc]))
    finally:
        dist.destroy_process_group()


def _grad_case():
    import numpy as np

    rng = np.random.default_rng(21)
    n = 120
    params = [np.stack([rng.uniform(-1, 1, n), rng.uniform(-0.7, 0.7, n), rng.uniform(3, 6, n)], 1),
              rng.normal(-2.6, 0.4, (n, 3)), rng.normal(0, 1, (n, 4)), rng.normal(0, 1, n),
              rng.normal(0, 0.3, (n, 16, 3))]
    cams = []
    for k in range(5):  # small views of uneven size around the cloud
        ang = 0.15 * (k - 2)
        R = np.array([[np.cos(ang), 0, -np.sin(ang)], [0, 1, 0], [np.sin(ang), 0, np.cos(ang)]])
        w, h = 64 + 16 * k, 48 + 8 * k
        cams.append(scenes.Camera(w, h, 0.8 * w, 0.8 * w, w / 2, h / 2, R, np.array([0.3 * (k - 2), 0.0, 0.2])))
    targets = [rng.uniform(0, 1, (c.height, c.width, 3)) for c in cams]
    return params, cams, targets


def test_two_rank_training_gradients_equal_one_rank():
    """Rendered gradients of 5 views split over two gloo ranks and summed by allreduce_gradients
    equal the one-rank sum over the same views (to the rounding of the order of the sum)."""
    import numpy as np

    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    params, cams, targets = _grad_case()
    R = oracle.Restatement()
    single = [np.zeros_like(p) for p in params]
    for k, cam in enumerate(cams):
        img = R.train_forward_f64(params, cam)
        for a, g in zip(single, R.train_backward_f64(params, cam, 2 * (img - targets[k]))):
            a += g
    assert sorted(out[0][1] + out[1][1]) == list(range(len(cams))) and out[0][1] and out[1][1]
    for rank, _, grads in out:
        for a, b in zip(grads, single):
            assert np.abs(b).max() > 0
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())
