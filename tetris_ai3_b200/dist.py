"""Multi-GPU plumbing, one process per GPU.

Evaluation (bench.py): each rank evaluates its own batch of sims (sims are
independent, so there is no data-path collective); the only communication is
the end-of-run reduction of device-timed seconds (max over ranks) and evaluated
placements (sum).

Training (island_group_score): a training run splits its islands into groups,
one per rank. Every rank keeps the whole (small) host state of the trainer --
all islands' optimisers, in lock step -- but scores only its own islands'
candidates; one all-gather of the per-game scores per generation then gives
every rank the full generation, so all ranks take identical optimiser steps and
the ring migration moves individuals between islands scored on different
ranks. The reference runs its islands on host threads, one evaluator each
(ta3_trainer/src/trainer2.cpp:98-100,144-170)."""
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


def island_group_score(local_score, islands: int, group=None):
    """A trainer score function (weights (n, P) float32, seeds (G,), max_moves ->
    scores (n, G), pieces (n, G)) for one rank of an island-group split: rows are
    island-major (n / islands per island); this rank scores islands i with
    i % world == rank through `local_score` and all-gathers the rest (the
    process group `group`, default the world). Without a process group it is
    `local_score` itself."""
    import numpy as np
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return local_score
    world, rank = dist.get_world_size(group), dist.get_rank(group)

    def score(w, seeds, max_moves):
        n = w.shape[0]
        if n % islands:
            raise ValueError("rows must be island-major with equal rows per island")
        rows, games = n // islands, len(seeds)
        mine = [i for i in range(islands) if i % world == rank]
        sc = np.zeros((n, games), np.float32)
        pc = np.zeros((n, games), np.uint32)
        if mine:
            idx = np.concatenate([np.arange(i * rows, (i + 1) * rows) for i in mine])
            res = local_score(np.ascontiguousarray(w[idx]), seeds, max_moves)
            s, p = res if isinstance(res, tuple) else (res, np.zeros((idx.size, games), np.uint32))
            sc[idx] = np.asarray(s, np.float32).reshape(idx.size, games)
            pc[idx] = np.asarray(p, np.uint32).reshape(idx.size, games)
        # each rank's islands' rows, bit patterns as int32; rank r's part supplies islands i % world == r
        t = torch.from_numpy(np.concatenate([sc.view(np.int32), pc.view(np.int32)], axis=1))
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        full_s = np.zeros((n, games), np.int32)
        full_p = np.zeros((n, games), np.int32)
        for r, part in enumerate(parts):
            a = part.numpy()
            for i in range(islands):
                if i % world == r:
                    full_s[i * rows:(i + 1) * rows] = a[i * rows:(i + 1) * rows, :games]
                    full_p[i * rows:(i + 1) * rows] = a[i * rows:(i + 1) * rows, games:]
        return full_s.view(np.float32), full_p.view(np.uint32)

    return score
