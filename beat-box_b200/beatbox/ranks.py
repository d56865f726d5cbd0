"""Host-side logic of multi-GPU runs (one process per GPU).

A single world does not shard: contacts cross any spatial split and the colour sweeps are
Gauss-Seidel over the whole contact graph, so N GPUs step N independent replicas.  Batches of
independent worlds do shard: `balanced_share` splits them over the ranks by body count.  Timings
are device times, reduced as the maximum over ranks (the job ends when the slowest rank does).
"""
from __future__ import annotations


def balanced_share(sizes, rank: int, world_size: int) -> list[int]:
    """Indices of the worlds that rank `rank` steps: greedy, largest world first, each to the
    rank with the fewest bodies so far (ties to the lowest rank).  Every world lands on exactly
    one rank, and every rank's index list is ascending."""
    load = [0] * world_size
    mine = []
    for k in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world_size), key=lambda r: (load[r], r))
        load[r] += int(sizes[k])
        if r == rank:
            mine.append(k)
    return sorted(mine)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks (the value itself without a process group)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: list[int] | int, max_seconds: float, world_size: int = 1) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    total = sum(units_per_rank) if isinstance(units_per_rank, list) else units_per_rank * world_size
    return total / max_seconds if max_seconds > 0 else 0.0
