"""Data-parallel helpers for multi-GPU tracing (one process per GPU, torch.distributed).

The path shards by views and samples: every rank holds the whole scene and traces its own
share of the views. The only exchange is the sum of the per-Gaussian material gradients and
the environment gradient after the adjoint, a single all-reduce of one flat buffer.
"""
from __future__ import annotations

import torch


def shard(count: int, rank: int, world: int) -> range:
    """Contiguous, balanced share of `count` items (views) for `rank` of `world`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_weighted(weights, rank: int, world: int) -> list:
    """The items (views) of `rank` of `world`, balanced by their weights (estimated path segments
    per view: its samples, or the segments its last trace counted): largest first, each to the
    least loaded rank (ties to the lower rank), which keeps the largest load within 4/3 of the best
    possible. Deterministic, so every rank computes the same assignment. Sorted item indices."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    w = [float(x) for x in weights]
    if any(x < 0 for x in w):
        raise ValueError("negative weight")
    load = [0.0] * world
    owner = [0] * len(w)
    for i in sorted(range(len(w)), key=lambda k: (-w[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += w[i]
    return [i for i in range(len(w)) if owner[i] == rank]


class GradientBucket:
    """A persistent flat buffer for the all-reduce of the step's gradients (material [N,5] and
    environment [He,We,4]): allocated at the first step, reused by every later one (no allocation
    inside a captured or timed step), with one all-reduce per step."""

    def __init__(self):
        self.flat = None

    def allreduce(self, grads, group=None):
        import torch.distributed as dist

        grads = [g for g in grads if g is not None and g.numel() > 0]
        total = sum(g.numel() for g in grads)
        if total == 0:
            return grads
        if self.flat is None or self.flat.numel() < total or self.flat.device != grads[0].device:
            self.flat = torch.empty(total, dtype=grads[0].dtype, device=grads[0].device)
        flat = self.flat[:total]
        off = 0
        for g in grads:
            flat[off:off + g.numel()].copy_(g.reshape(-1))
            off += g.numel()
        dist.all_reduce(flat, group=group)
        off = 0
        for g in grads:
            g.copy_(flat[off:off + g.numel()].view_as(g))
            off += g.numel()
        return grads


def allreduce_gradients(grads, group=None, flat: torch.Tensor | None = None):
    """Sum a list of gradient tensors over the process group with one all-reduce, in place.
    `flat` may hold a preallocated buffer of the total size (reused across steps)."""
    b = GradientBucket()
    b.flat = flat
    return b.allreduce(grads, group=group)
