"""Column sharding of Y = K~ W over ranks (one process per GPU).

The evaluation has no exchange step: right-hand sides are independent, so each rank
evaluates K~ on its own slab of W's columns with a full replica of the CDS, and the slabs
are gathered only if the caller wants Y everywhere.  No collective touches the data path
of the evaluation itself.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple


def column_range(nrhs: int, rank: int, world: int) -> Tuple[int, int]:
    """[start, stop) of rank's slab: contiguous, sizes differ by at most one."""
    if world < 1 or not (0 <= rank < world) or nrhs < 0:
        raise ValueError("bad rank / world / nrhs")
    base, extra = divmod(nrhs, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def sharded_apply(local_apply: Callable, W, group=None, gather: bool = True):
    """Apply `local_apply` (an (N, r_slab) -> (N, r_slab) map such as an Evaluator) to this
    rank's column slab of W (N, r), then all-gather the slabs into the full (N, r) result.
    With gather=False, returns (slab result, (start, stop))."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    n, r = W.shape
    start, stop = column_range(r, rank, world)
    Ys = local_apply(W[:, start:stop].contiguous()) if stop > start else W.new_zeros((n, 0))
    if not gather or world == 1:
        return Ys if world == 1 else (Ys, (start, stop))
    width = column_range(r, 0, world)[1]  # the widest slab; others are padded to it
    buf = W.new_zeros((n, width))
    buf[:, :stop - start] = Ys
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = W.new_empty((n, r))
    for k, p in enumerate(parts):
        a, b = column_range(r, k, world)
        out[:, a:b] = p[:, :b - a]
    return out
