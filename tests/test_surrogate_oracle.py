"""The surrogate's CPU checker (oracle/surrogate_oracle.py) pinned without a
GPU: its backward pass (rounding off) against central finite differences of
its own loss, its BF16 rounding against torch's, and its Spearman rank
correlation against scipy's."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import surrogate_oracle as so  # noqa: E402


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = so.init_params(1).astype(np.float64)
    x = rng.normal(size=(40, 97))
    y = rng.normal(size=40)
    g, _ = so.gradients(p, x, y, rounded=False)
    picks = list(rng.choice(so.NPARAM, 60, replace=False)) + [so.OFF_B3, so.OFF_B3 + 1, so.OFF_W3 + 5, so.OFF_B1 + 3]
    for i in picks:
        if so.OFF_W1 <= i < so.OFF_W2 and (i - so.OFF_W1) % so.IN_K >= so.IN:
            continue
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (so.loss_of(pp, x, y) - so.loss_of(pm, x, y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    v = np.random.default_rng(2).normal(size=10000).astype(np.float32) * 10 ** np.random.default_rng(3).uniform(
        -20, 20, 10000).astype(np.float32)
    ref = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(so.bf16(v), ref)


def test_spearman_matches_scipy():
    stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(4)
    a, b = rng.normal(size=200), rng.normal(size=200)
    b = a + 0.5 * b
    assert so.spearman(a, b) == pytest.approx(stats.spearmanr(a, b).statistic, abs=1e-12)
