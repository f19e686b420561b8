"""Multi-GPU use of the sweep: independent replicas only.

The checkerboard sweep of one lattice runs on one GPU; across GPUs the work
shards as independent lattices (one per rank, or a batch of replicas split
between ranks) with no collective on the data path.  The only cross-rank
operations are host-side bookkeeping: a barrier around timed regions and the
job-wide rate = all ranks' units / the slowest rank's time.
"""
from __future__ import annotations


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` of `world` (every item exactly once)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(items)[rank::world]


def job_rate(units_local: float, ms_local: float, dist=None, device=None):
    """(whole-job units per second, slowest rank's ms): units summed over the
    ranks, time the maximum over the ranks (torch.distributed if initialised)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return units_local / (ms_local * 1e-3), ms_local
    import torch

    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    u = torch.tensor([units_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()) / (float(t.item()) * 1e-3), float(t.item())
