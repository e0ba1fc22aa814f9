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
