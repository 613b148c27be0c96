"""Multi-GPU plumbing for evaluation: one process per GPU, each rank holding a
replica of the hierarchized grid and evaluating its own share of the query
points.  The evaluation itself needs no exchange; the only collectives are
for gathering results back in the caller's order and for timing (max over
ranks).  Works with any torch.distributed backend (NCCL on GPUs, gloo in the
CPU tests).
"""
from __future__ import annotations


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, start+count) share of `total` items for `rank`;
    the first total % world ranks get one extra item."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError(f"bad shard request total={total} rank={rank} world={world}")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def gather_in_order(local, total: int, group=None):
    """All-gathers every rank's contiguous shard (as produced by shard_range)
    into one tensor of `total` results in the original order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [shard_range(total, r, world)[1] for r in range(world)]
    width = max(counts) if counts else 0
    padded = torch.zeros(width, dtype=local.dtype, device=local.device)
    padded[: local.numel()] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)])


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest `value` over all ranks (device-timed step times are
    reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
