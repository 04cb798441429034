"""CMA-ES time-to-score: surrogate-assisted vs plain island training.

Workload: 4 islands x 50 candidates x 50 games, cap 2,000 pieces, dd-CMA-ES,
200 generations (20 iterations of 10, a new game seed every 10 iterations),
both runs from the same training seed, so both see the same game seeds.
The surrogate run fully evaluates generations 1-40; from generation 41 each
island samples 200 candidates, the GPU surrogate (97 -> 128 -> 128 -> 2,
tcgen05 kernels) ranks them, and the best 50 plus 5 random others are fully
evaluated; it is retrained every 10 generations and gated by Spearman rho >= 0.6
on the held-out latest generation. Every fitness comes from full evaluation.

The target score is the plain run's champion after 200 generations; the
metric is the surrogate run's wall-clock to first reach it, divided by the
plain run's wall-clock for its 200 generations (lower is better).

    python -m tetris_ai3_b200.time_to_score [--gens 200] [--out result.json]
"""
from __future__ import annotations

import argparse
import json
import math
import time

from . import trainer as T


def run(cfg, gens: int, label: str, log=print):
    tr = T.Trainer(cfg)
    t0 = time.perf_counter()
    traj = [{"gen": 0, "t": time.perf_counter() - t0, **_pick(tr.stats())}]
    per_iter = cfg.gens_per_iteration
    while tr.stats()["generation"] < gens:
        if tr.stats()["iteration"] % cfg.iterations_per_cycle == 0:
            tr.next_game_seed()
        tr.run_iteration()
        st = tr.stats()
        traj.append({"gen": st["generation"], "t": time.perf_counter() - t0, **_pick(st)})
        log(f"[{label}] gen {st['generation']:4d}  t {traj[-1]['t']:8.1f} s  best score {-st['best_fitness']:9.2f}"
            f"  rho {st['last_rho']:.3f}  active {st['surrogate_active']}", flush=True)
        assert per_iter > 0
    return traj, tr.stats()


def _pick(st):
    keys = ("best_fitness", "evaluations", "sims", "pieces", "eval_seconds", "host_seconds", "surrogate_seconds",
            "last_rho", "surrogate_active", "surrogate_trainings")
    return {k: (None if isinstance(st[k], float) and math.isnan(st[k]) else st[k]) for k in keys}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gens", type=int, default=200)
    ap.add_argument("--games", type=int, default=50)
    ap.add_argument("--cap", type=int, default=2000)
    ap.add_argument("--start", type=int, default=41)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)

    base = dict(islands=4, population=50, gens_per_iteration=10, iterations_per_cycle=10, games=args.games,
                max_moves=args.cap, algo=T.DD)
    plain_traj, plain_st = run(T.default_config(**base), args.gens, "plain")
    sur_cfg = T.default_config(**base, surrogate_start_gen=args.start, surrogate_sample=200, surrogate_top=50,
                               surrogate_random=5, surrogate_retrain=10, surrogate_min_rho=0.6)
    sur_traj, sur_st = run(sur_cfg, args.gens, "surrogate")

    target = plain_traj[-1]["best_fitness"]
    t_plain = plain_traj[-1]["t"]
    hit = next((p for p in sur_traj if p["best_fitness"] <= target), None)
    result = {
        "metric": "CMA-ES time-to-score, surrogate vs plain (4 islands x 50 x 50 games, cap 2000, "
                  f"{args.gens} generations)",
        "target_score": -target,
        "plain_seconds": t_plain,
        "surrogate_seconds_to_target": hit["t"] if hit else None,
        "surrogate_generation_at_target": hit["gen"] if hit else None,
        "ratio": (hit["t"] / t_plain) if hit else None,
        "goal_ratio": 0.5,
        "surrogate_final_score": -sur_traj[-1]["best_fitness"],
        "plain": plain_traj,
        "surrogate": sur_traj,
    }
    line = json.dumps({k: v for k, v in result.items() if k not in ("plain", "surrogate")})
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(result, f, indent=1)
    return result


if __name__ == "__main__":
    main()
