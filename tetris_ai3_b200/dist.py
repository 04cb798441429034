"""Multi-GPU plumbing for the evaluation path: one process per GPU, each rank
evaluates its own batch of sims (sims are independent, so there is no
data-path collective); the only communication is the end-of-run reduction of
device-timed seconds (max over ranks) and evaluated placements (sum)."""
from __future__ import annotations

import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment (1 process when absent)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def rank_seed(base_seed: int, rank: int) -> int:
    """The workload seed of a rank: rank r scores generation seeds base+r (weak scaling)."""
    return base_seed + rank


def reduce_timing(seconds: float, units: float, device=None):
    """Max of `seconds` and sum of `units` over all ranks (identity without a
    process group). Returns (max_seconds, total_units, units / max_seconds)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return seconds, units, units / seconds
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item()), float(u.item()) / float(t.item())
