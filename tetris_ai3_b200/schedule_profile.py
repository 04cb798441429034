"""Per-sim scheduling profile of one full generation (4 islands x 50 models x 50 games, cap 2000) on the GPU:
records when each sim started and finished and how many placements it
evaluated, and writes them to an .npz for analysis of the launch tail.

    python -m tetris_ai3_b200.schedule_profile --out profile.npz [--variant V]
"""
from __future__ import annotations

import argparse

import numpy as np

from . import ModelEvaluator, workload


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--variant", type=int, default=-1)
    args = ap.parse_args()
    b = workload.generation_batch()
    ev = ModelEvaluator()
    if args.variant >= 0:
        ev.select_variant(args.variant)
    ev.eval_timed(b.weights, b.seeds, b.max_moves)                     # warm-up
    sc, pc, ec, tm = ev.eval_timed(b.weights, b.seeds, b.max_moves)
    t0 = tm[:, 0].min()
    start = (tm[:, 0] - t0) / 1e6
    end = (tm[:, 1] - t0) / 1e6
    np.savez(args.out, start_ms=start, end_ms=end, pieces=pc, evals=ec, score=sc,
             launch=np.array([ev.launch_info()["grid"], ev.launch_info()["warps_per_block"]]))
    span = end.max()
    busy = (end - start).sum()
    warps = ev.launch_info()["grid"] * ev.launch_info()["warps_per_block"]
    print(f"makespan {span:.1f} ms, warp-busy fraction {busy / (span * warps):.3f}, "
          f"queue drained at {start.max():.1f} ms, longest sim {(end - start).max():.1f} ms "
          f"({pc[(end - start).argmax()]} pieces), placements {ec.sum():.3e}")


if __name__ == "__main__":
    main()
