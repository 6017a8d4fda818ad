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


def allreduce_gradients(grads, group=None, flat: torch.Tensor | None = None):
    """Sum a list of gradient tensors over the process group with one all-reduce, in place.
    `flat` may hold a preallocated buffer of the total size (reused across steps)."""
    import torch.distributed as dist

    grads = [g for g in grads if g is not None and g.numel() > 0]
    total = sum(g.numel() for g in grads)
    if total == 0:
        return grads
    if flat is None or flat.numel() < total or flat.device != grads[0].device:
        flat = torch.empty(total, dtype=grads[0].dtype, device=grads[0].device)
    off = 0
    for g in grads:
        flat[off:off + g.numel()].copy_(g.reshape(-1))
        off += g.numel()
    dist.all_reduce(flat[:total], group=group)
    off = 0
    for g in grads:
        g.copy_(flat[off:off + g.numel()].view_as(g))
        off += g.numel()
    return grads
