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

__all__ = ["views_for_rank", "views_per_rank", "allreduce_grads", "OverlappedGradSum"]


def views_for_rank(n_views: int, rank: int, world: int) -> list[int]:
    """Round-robin assignment of view indices to a rank."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return list(range(rank, n_views, world))


def views_per_rank(n_views: int, world: int) -> int:
    """The largest number of views any rank renders: the number of per-view
    reductions every rank issues (collectives must match across ranks)."""
    return -(-n_views // world)


class OverlappedGradSum:
    """Sum over ranks and views of per-view gradients, each view's reduction
    overlapping the rendering of the rank's next view.

    A rank renders its views one after another; after each view's backward it
    passes that view's gradients to ``add_view``, which packs them into one
    flat bucket and starts an asynchronous all-reduce (``async_op=True``; with
    NCCL it runs on the communicator's own stream while the next view's
    kernels run on the current one).  ``result`` waits for the reductions and
    returns the summed gradients.  At most ``in_flight`` buckets are pending;
    older ones are folded into the running total as new ones start.

    Every rank must call ``add_view`` the same number of times
    (``views_per_rank``): a rank with fewer views calls ``add_zero_view`` for
    the missing ones, so the collectives line up.  The total is the same sum
    as one all-reduce of each rank's accumulated gradients (up to the order
    of floating-point additions)."""

    def __init__(self, like, group=None, in_flight: int = 2):
        self.like = [t for t in like]
        self.shapes = [t.shape for t in self.like]
        self.numel = sum(t.numel() for t in self.like)
        self.group = group
        self.in_flight = max(1, int(in_flight))
        self.pending = []
        self.total = None
        self.views = 0

    def _start(self, flat):
        work = dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=self.group, async_op=True)
        self.pending.append((flat, work))
        self.views += 1
        while len(self.pending) > self.in_flight:
            self._fold()

    def _fold(self):
        flat, work = self.pending.pop(0)
        work.wait()
        if self.total is None:
            self.total = flat
        else:
            self.total.add_(flat)

    def add_view(self, grads) -> None:
        """Start the reduction of one view's gradients (tensors shaped like
        ``like``; None counts as zeros).  The tensors may be reused as soon
        as this returns: they are copied into the bucket."""
        parts = [(torch.zeros_like(t) if g is None else g).reshape(-1) for g, t in zip(grads, self.like)]
        self._start(torch.cat(parts))

    def add_zero_view(self) -> None:
        """This rank's share of a view it does not render: zeros."""
        t0 = self.like[0]
        self._start(torch.zeros(self.numel, dtype=t0.dtype, device=t0.device))

    def result(self):
        """Wait for every reduction; the summed gradients, shaped like ``like``."""
        while self.pending:
            self._fold()
        if self.total is None:
            return [torch.zeros_like(t) for t in self.like]
        out, off = [], 0
        for t in self.like:
            n = t.numel()
            out.append(self.total[off:off + n].view_as(t))
            off += n
        return out


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
