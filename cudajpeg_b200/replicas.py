"""Multi-GPU plumbing for the batch decoder: one process per GPU.

Images are independent, so the decode shards by image with no collective on
the data path.  Two layouts:

* weak scaling (default): rank r decodes its own batch, the mixed workload
  drawn with seed ``base_seed + r`` (rank 0's batch is the single-GPU one);
* strong scaling (``split``): one batch is partitioned across the ranks by
  pixel count (largest first onto the least-loaded rank).

Timing is the maximum over ranks of each rank's device time; the only
collectives are those reductions and barriers, outside the timed region.
"""
from __future__ import annotations

import os


def rank_env() -> tuple:
    """(rank, local_rank, world_size) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def rank_seed(base_seed: int, rank: int) -> int:
    """Workload seed of rank `rank` under weak scaling."""
    return base_seed + rank


def partition(weights, world: int) -> list:
    """Split item indices into `world` lists of near-equal total weight
    (longest-processing-time greedy; ties go to the lower rank).  Each list
    keeps ascending index order."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += weights[i]
    return [sorted(p) for p in parts]


def _reduce(value: float, dist, op, device) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, dist, device="cpu") -> float:
    """Maximum of `value` over all ranks (the job's time is its slowest rank)."""
    return _reduce(value, dist, dist.ReduceOp.MAX if dist else None, device)


def sum_over_ranks(value: float, dist, device="cpu") -> float:
    """Sum of `value` over all ranks (units processed by the whole job)."""
    return _reduce(value, dist, dist.ReduceOp.SUM if dist else None, device)
