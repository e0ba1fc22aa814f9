"""Several GPUs: one process per GPU, views (and scenes) as the independent units.

Rendering shards with no collective: the scene is replicated on every GPU and each rank renders its
share of the views (partition_views balances the shares by estimated cost: pixels plus Gaussians).
Training on one scene seen from views spread over the ranks has exactly one exchange step: each
rank's gradient buffers are summed with a single all_reduce (allreduce_gradients). Scenes that are
trained independently (one scene per rank) need no collective at all.

The reference has no multi-GPU path (its renderer drives one device, gpu_render.cu:267-375); this
module is the plumbing around the single-GPU library and holds no arithmetic of the path itself.
"""
from __future__ import annotations


def view_cost(width: int, height: int, gaussians: int) -> int:
    """Estimated work of one view: its pixels plus the Gaussians projected for it (the blend's
    work grows with the pixels, the projection's with the scene's Gaussians, and the two add)."""
    return int(width) * int(height) + int(gaussians)


def partition_views(costs, world: int) -> list[list[int]]:
    """Assigns view indices to `world` ranks, longest job first to the least-loaded rank.

    Deterministic (ties go to the lower view index and the lower rank), every view exactly once,
    and each rank's list in ascending view order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-int(costs[k]), k))
    load = [0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(k)
        load[r] += int(costs[k])
    return [sorted(s) for s in shares]


def my_views(cameras, gaussians: int, rank: int, world: int) -> list[int]:
    """This rank's view indices for a camera list rendered against one replicated scene."""
    costs = [view_cost(c.width, c.height, gaussians) for c in cameras]
    return partition_views(costs, world)[rank]


def allreduce_gradients(grads, group=None):
    """Sums gradient tensors over all ranks in place with one all_reduce of their concatenation."""
    import torch
    import torch.distributed as dist

    grads = [g for g in grads if g is not None]
    if not grads:
        return
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[off:off + n].view_as(g))
        off += n
