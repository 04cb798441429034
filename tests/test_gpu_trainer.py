"""The island trainer on the built-in GPU evaluator: every generation's
scores, hence every CMA-ES decision, equal those of the same trainer driven by
the oracle, so champions and optimiser means agree bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import oracle_eval

pytestmark = pytest.mark.gpu


def test_trainer_on_gpu_equals_trainer_on_oracle(host, oracle):
    cfg = dict(islands=3, population=6, gens_per_iteration=2, iterations_per_cycle=2, games=3, max_moves=120)

    def score(w, seeds, mm):
        sc, pc, _, _ = oracle_eval(oracle, w, seeds, mm)
        return sc.reshape(len(w), -1), pc.reshape(len(w), -1)

    gpu = host.Trainer(host.default_config(**cfg))
    cpu = host.Trainer(host.default_config(**cfg), score=score)
    gpu.run(3)
    cpu.run(3)
    for i in range(cfg["islands"]):
        xg, fg = gpu.champion(i)
        xc, fc = cpu.champion(i)
        assert fg == fc and np.array_equal(xg, xc)
        assert np.array_equal(gpu.island_mean(i), cpu.island_mean(i))
    sg, sc = gpu.stats(), cpu.stats()
    assert sg["pieces"] == sc["pieces"] and sg["sims"] == sc["sims"] and sg["best_fitness"] == sc["best_fitness"]


def test_widened_trainer_on_gpu_equals_trainer_on_oracle(host, oracle):
    """The trainer with the widened network (sep-CMA-ES, 4,929 parameters) on the
    GPU's widened kernel and on the oracle's widened restatement: same champions."""
    import ctypes as C
    from conftest import ptr
    cfg = dict(islands=2, population=6, gens_per_iteration=2, iterations_per_cycle=2, games=2, max_moves=60,
               algo=host.SEP, num_params=4929, sigma0=0.1)

    def score(w, seeds, mm):
        w = np.ascontiguousarray(w, np.float32)
        s = np.ascontiguousarray(seeds, np.uint64)
        n = len(w) * len(s)
        sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        ev = C.c_uint64()
        oracle.ta3o_eval_net_mt(ptr(w), 64, 64, len(w), ptr(s), len(s), mm, 8, ptr(sc), ptr(pc), ptr(lc),
                                C.byref(ev))
        return sc.reshape(len(w), -1), pc.reshape(len(w), -1)

    gpu = host.Trainer(host.default_config(**cfg))
    cpu = host.Trainer(host.default_config(**cfg), score=score)
    gpu.run(2)
    cpu.run(2)
    for i in range(cfg["islands"]):
        xg, fg = gpu.champion(i)
        xc, fc = cpu.champion(i)
        assert fg == fc and np.array_equal(xg, xc)
    assert gpu.stats()["pieces"] == cpu.stats()["pieces"]


@pytest.mark.parametrize("num_params", [97, 4929])
def test_built_in_gpu_surrogate_prescreens(host, num_params):
    """The trainer's own GPU surrogate (97 -> 128 -> 128 -> 2 for v11, 4929 -> 256 ->
    256 -> 2 for the widened vector) on a quadratic landscape: it retrains on the
    archive and gates itself on held-out rank correlation; the 97-parameter model
    passes the gate and pre-screens the later generations."""
    target = np.linspace(-0.5, 0.5, num_params)

    def score(w, seeds, mm):
        base = -((w.astype(np.float64) - target) ** 2).sum(1)
        return (base[:, None] + np.zeros(len(seeds))[None, :]).astype(np.float32)

    cfg = host.default_config(islands=2, population=16, gens_per_iteration=3, iterations_per_cycle=2, games=2,
                              max_moves=50, algo=host.SEP, num_params=num_params, sigma0=0.3,
                              surrogate_start_gen=6, surrogate_sample=32, surrogate_top=8, surrogate_random=2,
                              surrogate_retrain=2, surrogate_min_rho=0.3, surrogate_epochs=30, surrogate_batch=64)
    t = host.Trainer(cfg, score=score)
    for _ in range(10):
        t.run_generation()
    st = t.stats()
    assert st["surrogate_trainings"] >= 2 and np.isfinite(st["last_rho"])
    sizes = [n for n, _, _ in t.calls]
    assert sizes[:6] == [2 * 16] * 6                 # start-up and generations 1..5: full evaluation
    assert set(sizes[6:]) <= {2 * 16, 2 * 10}        # then full, or pre-screened (8 + 2 per island)
    if num_params == 97:                             # the small model learns this landscape and screens
        assert st["surrogate_active"] == 1 and 2 * 10 in sizes[6:]
