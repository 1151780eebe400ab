"""Several GPUs: independent replicas, no collective on the data path.

The right-hand side needs no communication between basins, so N GPUs run N
copies of a workload (or N disjoint subsets of an ensemble's members), one
process per GPU.  Only the timing is reduced: the whole-job throughput is all
ranks' work divided by the slowest rank's time.
"""
from __future__ import annotations


def reduce_throughput(elapsed_ms: float, units: float, world: int, device=None):
    """(slowest rank's elapsed ms, sum of all ranks' units) over the default
    process group; the local pair when world == 1."""
    if world == 1:
        return float(elapsed_ms), float(units)
    import torch
    import torch.distributed as dist
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def member_share(count: int, rank: int, world: int) -> list:
    """Indices of the ensemble members rank `rank` of `world` runs: a
    round-robin split, disjoint and covering 0 .. count-1."""
    return list(range(rank, count, world))
