"""Sharding trajectories (or models) across ranks, one process per GPU.

Trajectories are independent and every random number is keyed by the
global trajectory id, so a shard is just a contiguous id range: results do
not depend on how the work is split, and the data path has no collective.
The only cross-rank traffic is bookkeeping: timing (max over ranks) and
event counts (sum), via ``torch.distributed`` (NCCL on GPUs, gloo on CPU).
"""


def shard_range(n_total, rank, world):
    """(first id, count) of rank's contiguous share of n_total items."""
    base, extra = divmod(int(n_total), int(world))
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def shard_items(items, rank, world):
    start, count = shard_range(len(items), rank, world)
    return items[start:start + count], start


def reduce_time_and_count(ms, count, device=None):
    """(max of ms over ranks, sum of count over ranks); identity when
    torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), float(count)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())
