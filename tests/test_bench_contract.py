"""bench.py's output contract: one JSON line with the keys the driver reads.

CPU: the reference arm (the reference's own CPU path, timed on the host cores) on a short sample.
GPU: the evaluator's arm on a small generation (5,000 sims, cap 40): metric, timing, clocks,
roofline, CPU baseline slot, end-to-end figure and the launch count."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(*args, timeout=600):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def _check_common(d):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "e2e"):
        assert k in d, k
    assert d["unit"] == "placements/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"]
    assert d["e2e"]["unit"] == d["unit"] and d["e2e"]["value"] > 0


def test_reference_arm_prints_its_line():
    d = _run("--impl", "reference", "--steps", "1", "--warmup", "3", "--ref-budget", "0.5")
    _check_common(d)
    assert d["impl"] == "reference"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


@pytest.mark.gpu
def test_evaluator_arm_prints_its_line():
    d = _run("--islands", "1", "--pop", "100", "--games", "50", "--cap", "40", "--steps", "2", "--warmup", "3",
             "--no-cpu-baseline", "--no-autotune")
    _check_common(d)
    assert "impl" not in d and d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    assert d["ms_per_step"] > 0 and d["cpu_baseline"] is None
    r = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert r["bound"] == "issue" and 0 < r["frac"] and r["peak"] > 0
    assert set(r["ncu_full_occupancy"]) == {"issue_slots_busy", "warp_execution_efficiency",
                                            "shared_memory_throughput"}
    c = d["clocks"]
    assert c["sm_mhz"] > 0 and c["sm_max_mhz"] > 0 and isinstance(c["reasons"], list)
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    # 5,000 sims fill the grid: the single-warp kernel and the hand-off's paired kernel per step
    assert d["gpu_launches"] == 2 * d["steps"]
    assert d["config"]["launch"]["kernels"] == 2
