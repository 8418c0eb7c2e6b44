"""Data-parallel multi-view rendering over several GPUs (one process each).

The path shards by view: given replicated vertices, indices and cell values,
each view's projection, lists and blend are independent, so every rank
renders its own views with no data-path collective.  Training has one
exchange step, the sum over views of the vertex and cell-value gradients
(12 V + 28 T bytes), done as one NCCL all-reduce over a flat bucket
(``torch.distributed`` with the "nccl" backend on GPUs; "gloo" works the same
on CPU tensors).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

__all__ = ["views_for_rank", "allreduce_grads"]


def views_for_rank(n_views: int, rank: int, world: int) -> list[int]:
    """Round-robin assignment of view indices to a rank."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return list(range(rank, n_views, world))


def allreduce_grads(tensors, group=None) -> None:
    """Sum `tensors` over all ranks in place, as one flat bucket (one
    collective per call, the same on every rank)."""
    tensors = [t for t in tensors if t is not None]
    if not tensors:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n
