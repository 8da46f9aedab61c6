"""Multi-GPU replicas: one process per GPU, each with the full geometry and
tables, simulating a disjoint share of the primaries.

Primaries are independent, so there is no data-path collective: each rank
pushes its contiguous share with the global primary index as its random-
stream base (nbx_set_uid_base), which makes every electron's stream, and so
the combined result, independent of the number of ranks.  The only
collective is the final sum of the per-pixel FP64 accumulators."""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """Contiguous [start, stop) share of n items for this rank."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def run_shard(ctx, records, rank: int, world: int, n_pixels: int, nx: int):
    """Simulate this rank's share of `records` (.pri records) on ctx and
    return its per-pixel FP64 accumulators (n_pixels x 5)."""
    start, stop = shard_range(len(records), rank, world)
    part = records[start:stop]
    ctx.set_uid_base(start)
    ctx.reset_tallies()
    ctx.set_tag_range(max(len(part), 1))
    if len(part):
        ctx.push_records(part)
        ctx.run()
    pixel_of_tag = (part["py"].astype(np.uint32) * nx + part["px"].astype(np.uint32))
    return ctx.pixel_yields(pixel_of_tag, n_pixels) if len(part) else np.zeros((n_pixels, 5))


def reduce_pixel_yields(dist, yields: np.ndarray) -> np.ndarray:
    """Sum the per-pixel accumulators over ranks (process group `dist`, any
    backend; None = single process).  The caller's array is left unchanged:
    the all-reduce works on a copy."""
    if dist is None:
        return yields
    import torch
    t = torch.tensor(np.asarray(yields, np.float64))
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()
