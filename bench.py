"""Benchmark: beam placements/s of one CMA-ES generation's evaluation on B200.

One step = one CMA-ES generation: 4 islands x 50 candidates x 50 games =
10,000 (model, game) sims, v11 weights, cap 2,000 pieces, every game played
with the depth-4 beam (16/32/32) to the cap or top-out. The unit is the
evaluated beam placement (one value-model call inside search_move_beam), an
algorithmic count that is identical on GPU and CPU because the decisions are
bit-identical.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       value: kernel-only, inputs resident in HBM, CUDA events on the launch
           stream, L2 flushed between timed steps; e2e: the public API
           (ta3b_eval_islands) from pinned host buffers, copies included.
reference  the reference's own CPU path (oracle/_ref, compiled from the
           reference sources) on all host threads, bounded sample per step.
For N > 1 (torchrun) every rank evaluates its own generation (weak scaling,
no data-path collective); value = all ranks' placements / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tetris_ai3_b200 import workload  # noqa: E402

METRIC = "beam placements/s on 1 B200 (one CMA-ES generation: 4 islands x 50 models x 50 games = 10k sims, cap 2000)"
UNIT = "placements/s"
# Issue roofline (the path is INT32/FP32 issue-bound, not HBM- or tensor-bound):
# REF_OPS_PER_PLACEMENT is the reference algorithm's operation count for one
# evaluated placement, counted on the restatement: drop/collision over 10 columns
# (230) + lock (80) + full-row test (12) + clear histogram (3); v11 features
# (16 + 46 per column x 10 + 11); MLP 8 x (10 mul + 10 add + relu) + 8 mul + 8 add
# (192); key (6) = 1010.
REF_OPS_PER_PLACEMENT = 1010
# The widened 10 -> 64 -> 64 -> 1 network replaces the MLP's 192 by
# 64 x (10 mul + 10 add + relu) + 64 x (64 mul + 64 add + relu) + 64 mul + 64 add = 9,728.
REF_OPS_PER_PLACEMENT_WIDE = 1010 - 192 + 9728
# width 32: 32 x (10 mul + 10 add + relu) + 32 x (32 mul + 32 add + relu) + 32 mul + 32 add = 2,816
REF_OPS_PER_PLACEMENT_WIDE32 = 1010 - 192 + 2816
METRIC_STRESS = ("beam placements/s on 1 B200 (uneven-length stress: 200 models x 100 games = 20k sims, "
                 "10% v11 champion, cap 10000)")
METRIC_WIDE = ("beam placements/s on 1 B200 (widened 10-64-64-1 evaluator: 8 islands x 100 models x 100 games "
               "= 80k sims, cap 2000)")
METRIC_WIDE32 = ("beam placements/s on 1 B200 (widened 10-32-32-1 evaluator: 8 islands x 100 models x 100 games "
                 "= 80k sims, cap 2000)")
METRICS = {"wide": METRIC_WIDE, "wide32": METRIC_WIDE32, "stress": METRIC_STRESS}
HIDDEN = {"wide": 64, "wide32": 32}           # the widened models' hidden width
# What the single-warp kernel executes per placement (ncu thread_inst_executed / placements, on a
# full-occupancy capture) and the DRAM bytes of one full-generation evaluation (ncu
# dram__bytes_read.sum + dram__bytes_write.sum of its two launches, 1-pass capture).
LANE_INSTR_PER_PLACEMENT = 541
# The three counters the path is judged by, from the same kind of capture of the hand-off flavour
# the bench runs (ncu --set full at full occupancy): issue slots busy
# (smsp__issue_active.avg.pct_of_peak_sustained_active), warp execution efficiency
# (smsp__thread_inst_executed_per_inst_executed.ratio / 32) and shared-memory throughput
# (l1tex__data_pipe_lsu_wavefronts_mem_shared.sum.pct_of_peak_sustained_elapsed).
NCU_FULL_OCCUPANCY = {"issue_slots_busy": 0.626, "warp_execution_efficiency": 0.878,
                      "shared_memory_throughput": 0.185}
DRAM_BYTES_PER_LAUNCH = 1_181_184


from tetris_ai3_b200.dist import rank_env as _dist_env, rank_seed, reduce_timing  # noqa: E402


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace('.', '').isdigit())
                if any(r[3].replace('.', '').isdigit() for r in rows) else None}


def _ref_lib(hidden: int = 0):
    """The reference's CPU path (oracle/_ref) if built, else the oracle's restatement,
    as (batch function with the ta3ref_eval_mt signature, kind); hidden = 0 for v11,
    else the widened network's width (64 or 32)."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libta3ref.so")
    if os.path.exists(ref):
        lib = C.CDLL(ref)
        fn = {0: lib.ta3ref_eval_mt, 64: lib.ta3ref_eval_wide_mt, 32: lib.ta3ref_eval_wide32_mt}[hidden]
        return fn, "reference"
    port = os.path.join(ROOT, "oracle", "_build", "libta3oracle.so")
    if not os.path.exists(port):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    lib = C.CDLL(port)
    if hidden:
        return (lambda *a: lib.ta3o_eval_net_mt(a[0], hidden, hidden, *a[1:])), "port"
    return lib.ta3o_eval_mt, "port"


def cpu_rate(batch: workload.Batch, budget_s: float, threads: int):
    """Placements/s of the CPU path over a bounded sample of the batch: island 0's
    (model, game) pairs in workload order, `threads` games of one model per call
    (one host thread each), until budget_s of work."""
    f, kind = _ref_lib({workload.NUM_PARAMS_WIDE: 64, workload.NUM_PARAMS_WIDE32: 32}.get(batch.weights.shape[1], 0))
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    games = batch.games
    mpi = batch.models // batch.islands
    total_ev, sims, t_used = 0, 0, 0.0
    m, g0 = 0, 0
    while t_used < budget_s and m < mpi:
        c = min(threads, games - g0)
        w = np.ascontiguousarray(batch.weights[m:m + 1], np.float32)
        seeds = np.ascontiguousarray(batch.seeds[0][g0:g0 + c], np.uint64)
        sc = np.zeros(c, np.float32)
        evs = C.c_uint64()
        t0 = time.perf_counter()
        f(p(w), C.c_uint32(1), p(seeds), C.c_uint32(c), C.c_uint32(batch.max_moves), C.c_uint32(c), p(sc),
          None, None, C.byref(evs))
        t_used += time.perf_counter() - t0
        total_ev += evs.value
        sims += c
        g0 += c
        if g0 >= games:
            m, g0 = m + 1, 0
    return total_ev / t_used, kind, sims, t_used


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _batch(args, rank: int = 0) -> workload.Batch:
    """The workload of one rank (weak scaling: rank r scores generation seed base+r)."""
    if args.model == "stress":
        return workload.uneven_batch(models=args.pop or 200, games=args.games or 100, max_moves=args.cap or 10000,
                                     seed=rank_seed(2, rank))
    if args.model in HIDDEN:
        return workload.wide_batch(islands=args.islands or 8, pop=args.pop or 100, games=args.games or 100,
                                   max_moves=args.cap or 2000, seed=rank_seed(3, rank), hidden=HIDDEN[args.model])
    return workload.generation_batch(islands=args.islands or 4, pop=args.pop or 50, games=args.games or 50,
                                     max_moves=args.cap or 2000, seed=rank_seed(1, rank))


def run_reference(args):
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    batch = _batch(args)
    metric = METRICS.get(args.model, METRIC)
    threads = host_threads()
    rates = []
    kind = "reference"
    sample_desc = ""
    for step in range(args.warmup + args.steps):
        r, kind, sims, t = cpu_rate(batch, budget_s=args.ref_budget, threads=threads)
        if step >= args.warmup:
            rates.append(r)
            sample_desc = (f"first {sims} sims of the generation (island 0, model-major), cap {batch.max_moves}, "
                           f"{t:.1f} s per step")
    v = float(np.mean(rates))
    line = {"impl": "reference", "metric": metric, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32+int32", "data": "synthetic",
            "config": {"workload": batch.name, "global_batch": batch.sims, "seq_len": batch.max_moves,
                       "parallelism": f"{threads} host threads", "cpu": _cpu_model()},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample_desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_ours(args):
    import torch
    import torch.distributed as dist
    from tetris_ai3_b200 import ModelEvaluator

    rank, world, local = _dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    # weak scaling: each rank scores its own generation (islands seeded per rank)
    batch = _batch(args, rank)
    wide = args.model in HIDDEN
    metric = METRICS.get(args.model, METRIC)
    ops_per_placement = {"wide": REF_OPS_PER_PLACEMENT_WIDE, "wide32": REF_OPS_PER_PLACEMENT_WIDE32}.get(
        args.model, REF_OPS_PER_PLACEMENT)
    ev = ModelEvaluator(device=local)
    stream = torch.cuda.Stream(device=dev)
    w_dev = torch.from_numpy(batch.weights).to(dev)
    s_dev = torch.from_numpy(batch.seeds.view(np.int64)).to(dev)
    n = batch.sims
    score = torch.empty(n, dtype=torch.float32, device=dev)
    pieces = torch.empty(n, dtype=torch.int32, device=dev)
    lines = torch.empty(n, dtype=torch.int32, device=dev)
    evals = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)   # > 126 MB L2
    torch.cuda.synchronize()

    def step():
        ev.eval_device(w_dev, s_dev, batch.max_moves, score, pieces, lines, evals, num_islands=batch.islands,
                       stream=stream)

    tune = None
    if args.variant >= 0:
        ev.select_variant(args.variant)
    elif not args.no_autotune and not wide:
        tune = ev.autotune(w_dev, s_dev, batch.max_moves, score, pieces, lines, evals, batch.islands, stream)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = []
    placements = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            with torch.cuda.stream(stream):
                step()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
            placements += int(evals.to(torch.int64).sum().item())
    torch.cuda.synchronize()
    kernels_per_step = ev.launch_info()["kernels"]    # 2 when the tail hand-off's paired kernel ran
    clocks = clk.summary()
    t_local = sum(ms) / 1000.0
    t_max, total_pl, value = reduce_timing(t_local, float(placements), dev)

    # ---- end to end through the public API: pinned host buffers in, host results out
    h_w = torch.from_numpy(batch.weights).pin_memory()
    h_s = torch.from_numpy(batch.seeds.view(np.int64)).pin_memory()
    h_sc = torch.empty(n, dtype=torch.float32).pin_memory()
    h_pc = torch.empty(n, dtype=torch.int32).pin_memory()
    h_lc = torch.empty(n, dtype=torch.int32).pin_memory()
    lib = ev._lib
    vp = lambda t: C.c_void_p(t.data_ptr())
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        rc = lib.ta3b_eval_islands(ev._ctx, vp(h_w), batch.islands, batch.models // batch.islands,
                                   batch.weights.shape[1], vp(h_s),
                                   batch.games, batch.max_moves, vp(h_sc), vp(h_pc), vp(h_lc))
        if rc:
            raise RuntimeError(lib.ta3b_last_error(ev._ctx).decode())
    e2e_t, _, _ = reduce_timing(time.perf_counter() - t0, 0.0, dev)
    assert h_sc.numpy().tobytes() == score.cpu().numpy().tobytes(), "e2e results differ from the device run"
    e2e_value = (total_pl / args.steps) * e2e_steps / e2e_t
    h2d = batch.weights.nbytes + batch.seeds.nbytes
    d2h = n * (4 + 4 + 4)

    if rank == 0:
        peaks, kind = _peaks()
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
        peak_issue = sms * 4 * 32 * sm_mhz * 1e6 / 1e12            # lane-instructions, T/s
        per_gpu = value / world
        ach = per_gpu * ops_per_placement / 1e12
        roof = {"bound": "issue", "achieved": ach, "peak": peak_issue, "unit": "T int32/fp32 lane-ops/s",
                "frac": ach / peak_issue, "traffic": DRAM_BYTES_PER_LAUNCH,
                "peak_source": f"{sms} SMs x 4 schedulers x 32 lanes x sm_max_mhz {sm_mhz:.0f} "
                               f"(MEASURED_PEAKS.json, {kind})",
                "ops_per_placement": ops_per_placement,
                "ops_basis": "placements/s of the whole evaluation (with the tail hand-off, the single-warp "
                             "kernel and the paired kernel that finishes its last games); frac (the headline) counts "
                             "the reference algorithm's operations per placement (an algorithmic count, hand count "
                             "above); frac_executed counts the lane-instructions the single-warp kernel executes per "
                             "placement at full occupancy (ncu thread_inst_executed / placements)",
                "lane_instr_per_placement_measured": None if wide else LANE_INSTR_PER_PLACEMENT,
                "frac_executed": None if wide else per_gpu * LANE_INSTR_PER_PLACEMENT / 1e12 / peak_issue,
                "ncu_full_occupancy": None if wide else NCU_FULL_OCCUPANCY}
        if wide:
            roof["traffic"] = None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = host_threads()
            r, ck, sims, t = cpu_rate(batch, budget_s=args.cpu_budget, threads=threads)
            cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": ck,
                   "sample": f"first {sims} sims of the generation (island 0, model-major), cap {batch.max_moves}, "
                             f"{t:.1f} s"}
        line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp32+int32", "data": "synthetic",
                "config": {"workload": batch.name, "global_batch": batch.sims * world, "seq_len": batch.max_moves,
                           "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                           "l2": "flushed (256 MB write) between timed steps",
                           "launch": ev.launch_info(),
                           "autotune_ms": tune},
                "sims_per_step": batch.sims, "placements_per_step": total_pl / args.steps / world,
                "clocks": clocks, "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": e2e_steps},
                # per step: the evaluation kernels (the single-warp kernel and, with the tail
                # hand-off, the paired kernel that finishes its tail; the widened model adds its
                # weight-repack kernel)
                "gpu_launches": args.steps * (kernels_per_step + (1 if wide else 0))}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=-1, help="fixed kernel variant (default: autotune)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--model", choices=["v11", "wide", "wide32", "stress"], default="v11",
                    help="v11 (headline), the widened 10-64-64-1 (wide) or 10-32-32-1 (wide32) evaluator's "
                         "80k-sim generation, or the uneven-length stress batch (20k sims, 10%% champion, cap 10000)")
    # reduced shapes for profiling captures only (the headline is the default full generation)
    ap.add_argument("--islands", type=int, default=0)
    ap.add_argument("--pop", type=int, default=0)
    ap.add_argument("--games", type=int, default=0)
    ap.add_argument("--cap", type=int, default=0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
