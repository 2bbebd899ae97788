"""Batch sharding across GPUs (one process per GPU).

Rows of a batched transform are independent, so a batch is split into contiguous row ranges,
one per rank, and every rank transforms its own range in its own HBM with no data-path
collective.  An optional gather assembles the full result on every rank with one all-gather of
equal-sized, padded shards (plain NCCL / gloo all_gather into local buffers).
"""
from __future__ import annotations


def shard_rows(batch: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [start, stop) row range of `rank`; the first batch % world ranks get one
    extra row, so sizes differ by at most one and every row is covered exactly once."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("invalid world/rank")
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def sharded_fft(x, fn, group=None, gather: bool = False):
    """Apply the row-wise transform `fn` to this rank's shard of x ([batch, ...], identical on
    all ranks) and optionally all-gather the shards.  Returns (local_result, full_or_None)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    start, stop = shard_rows(x.shape[0], world, rank)
    local = fn(x[start:stop])
    if not gather or world == 1:
        return local, (local if gather else None)
    rows = -(-x.shape[0] // world)   # padded shard size
    pad = torch.zeros((rows,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    full = torch.cat([p[: shard_rows(x.shape[0], world, r)[1] - shard_rows(x.shape[0], world, r)[0]]
                      for r, p in enumerate(parts)])
    return local, full
