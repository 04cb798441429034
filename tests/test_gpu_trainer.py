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
