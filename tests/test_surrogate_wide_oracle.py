"""The layer-by-layer surrogate's CPU checker (oracle/surrogate_wide_oracle.py)
pinned without a GPU: its backward pass (rounding off) against central finite
differences of its own loss at small and padded sizes, and its layout against
the v11 checker where the two models coincide except for the output layer's
gradient rounding."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import surrogate_oracle as so  # noqa: E402
import surrogate_wide_oracle as sw  # noqa: E402


@pytest.mark.parametrize("in_dim,hidden", [(37, 128), (130, 256)])
def test_backward_matches_finite_differences(in_dim, hidden):
    d = sw.Dims(in_dim, hidden)
    rng = np.random.default_rng(in_dim)
    p = sw.init_params(d, 1).astype(np.float64)
    x = rng.normal(size=(30, in_dim))
    y = rng.normal(size=30)
    g, _ = sw.gradients(d, p, x, y, rounded=False)
    picks = list(rng.choice(d.n, 60, replace=False)) + [d.b3, d.b3 + 1, d.w3 + 5, d.b1 + 3, d.w2 + 7]
    checked = 0
    for i in picks:
        if d.w1 <= i < d.w2 and (i - d.w1) % d.inp >= d.in_dim:
            assert g[i] == 0.0            # padding columns get no gradient
            continue
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (sw.loss_of(d, pp, x, y) - sw.loss_of(d, pm, x, y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
        checked += 1
    assert checked > 40


def test_layout_and_forward_agree_with_the_v11_checker():
    """At in_dim 97, hidden 128 the two checkers describe the same network: same
    forward outputs once the parameters are moved between the two layouts."""
    d = sw.Dims(97, 128)
    rng = np.random.default_rng(2)
    p11 = so.init_params(4)
    pw = np.zeros(d.n, np.float32)
    w1, w2, w3, b1, b2, b3 = so.unpack(p11)
    pw[d.w1:d.w2].reshape(128, d.inp)[:, :97] = w1
    pw[d.w2:d.w3] = w2.reshape(-1)
    pw[d.w3:d.b1] = w3.reshape(-1)
    pw[d.b1:d.b2], pw[d.b2:d.b3], pw[d.b3:] = b1, b2, b3
    x = rng.normal(size=(50, 97)).astype(np.float32)
    a, _ = so.forward(p11, x)
    b, _ = sw.forward(d, pw, x)
    assert np.allclose(a, b, rtol=1e-6, atol=1e-6)
