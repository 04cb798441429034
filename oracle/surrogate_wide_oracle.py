"""CPU checker for the layer-by-layer surrogate (tetris_ai3_b200/csrc/ta3s_wide.cu,
the ta3w_* functions of include/ta3b_surrogate.h).

Test infrastructure only: imported by tests/, never by the product. No
counterpart in the reference; this restates the model the kernels compute --
in_dim -> H -> H -> 2, ReLU, Gaussian NLL 0.5 * (s + (y - mu)^2 exp(-s)) with s
clamped to [-12, 12], averaged over the batch -- in float64, with BF16 rounding
(nearest even) exactly where the kernels round:
  standardised inputs X, W1, W2, relu(H1), dH2, dH1 (masked).
Everything else is FP32 on the GPU (the output layer, the loss, dmu / ds, dW3,
the bias gradients), so the checker keeps those in float64 (dmu / ds rounded to
float32 like the kernels' values).
Parameter layout: W1 [H][INP] (INP = in_dim rounded up to 128, padding columns
zero), W2 [H][H], W3 [2][H], b1 [H], b2 [H], b3 [2].
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from surrogate_oracle import _bf16, spearman  # noqa: F401  (re-exported for the tests)


@dataclass(frozen=True)
class Dims:
    in_dim: int
    hidden: int

    @property
    def inp(self) -> int:
        return (self.in_dim + 127) // 128 * 128

    @property
    def w1(self) -> int:
        return 0

    @property
    def w2(self) -> int:
        return self.hidden * self.inp

    @property
    def w3(self) -> int:
        return self.w2 + self.hidden * self.hidden

    @property
    def b1(self) -> int:
        return self.w3 + 2 * self.hidden

    @property
    def b2(self) -> int:
        return self.b1 + self.hidden

    @property
    def b3(self) -> int:
        return self.b2 + self.hidden

    @property
    def n(self) -> int:
        return self.b3 + 2


def unpack(d: Dims, p: np.ndarray):
    p = np.asarray(p)
    w1 = p[d.w1:d.w2].reshape(d.hidden, d.inp)[:, :d.in_dim]
    w2 = p[d.w2:d.w3].reshape(d.hidden, d.hidden)
    w3 = p[d.w3:d.b1].reshape(2, d.hidden)
    return w1, w2, w3, p[d.b1:d.b2], p[d.b2:d.b3], p[d.b3:d.n]


def init_params(d: Dims, seed: int = 0, bias: float = 0.1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(d.n, np.float32)
    p[d.w1:d.w2].reshape(d.hidden, d.inp)[:, :d.in_dim] = rng.uniform(-1, 1, (d.hidden, d.in_dim)) * np.sqrt(
        6 / d.in_dim)
    p[d.w2:d.w3] = rng.uniform(-1, 1, d.hidden * d.hidden) * np.sqrt(6 / d.hidden)
    p[d.w3:d.b1] = rng.uniform(-1, 1, 2 * d.hidden) * np.sqrt(1 / d.hidden)
    p[d.b1:d.b3] = rng.uniform(-bias, bias, 2 * d.hidden)
    p[d.b3:] = rng.uniform(-bias, bias, 2)
    return p


def _exact(a):
    return np.asarray(a, dtype=np.float64)


def forward(d: Dims, p: np.ndarray, x: np.ndarray, rounded: bool = True):
    """(mean, log-variance) per row and the intermediates of the backward pass.
    rounded=False drops every BF16 / FP32 rounding (for finite differences)."""
    bf16 = _bf16 if rounded else _exact
    p = np.asarray(p, np.float32 if rounded else np.float64)
    w1, w2, w3, b1, b2, b3 = (np.asarray(t, np.float64) for t in unpack(d, p))
    xb = bf16(x)
    h1b = bf16(np.maximum(xb @ bf16(w1).T + b1, 0.0))
    z2 = h1b @ bf16(w2).T + b2
    h2 = np.maximum(z2, 0.0)
    out = h2 @ w3.T + b3
    return out, dict(xb=xb, h1b=h1b, z2=z2, h2=h2, w2=w2, w3=w3)


def gradients(d: Dims, p: np.ndarray, x: np.ndarray, y: np.ndarray, rounded: bool = True):
    """Gradient of the mean NLL (parameter layout) and the summed loss."""
    bf16 = _bf16 if rounded else _exact
    f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if rounded else _exact
    out, c = forward(d, p, x, rounded)
    n = len(x)
    mu, s_raw = out[:, 0], out[:, 1]
    s = np.clip(s_raw, -12.0, 12.0)
    e = np.exp(-s)
    dy = np.asarray(y, np.float64) - mu
    loss = float(np.sum(0.5 * (s + dy * dy * e)))
    dmu = f32(-dy * e / n)
    ds = f32(np.where((s_raw > -12) & (s_raw < 12), 0.5 * (1 - dy * dy * e) / n, 0.0))
    g = np.zeros(d.n, np.float64)
    g[d.w3:d.b1] = np.concatenate([c["h2"].T @ dmu, c["h2"].T @ ds])
    g[d.b3] = dmu.sum()
    g[d.b3 + 1] = ds.sum()
    dh2b = bf16(np.where(c["z2"] > 0, dmu[:, None] * c["w3"][0] + ds[:, None] * c["w3"][1], 0.0))
    g[d.b2:d.b3] = dh2b.sum(0)
    g[d.w2:d.w3] = (dh2b.T @ c["h1b"]).reshape(-1)
    dh1b = bf16(np.where(c["h1b"] > 0, dh2b @ bf16(c["w2"]), 0.0))
    g[d.b1:d.b2] = dh1b.sum(0)
    gw1 = np.zeros((d.hidden, d.inp))
    gw1[:, :d.in_dim] = dh1b.T @ c["xb"]
    g[d.w1:d.w2] = gw1.reshape(-1)
    return g, loss


def loss_of(d: Dims, p: np.ndarray, x: np.ndarray, y: np.ndarray, rounded: bool = False) -> float:
    """Mean NLL (for finite differences)."""
    out, _ = forward(d, p, x, rounded)
    s = np.clip(out[:, 1], -12.0, 12.0)
    dy = np.asarray(y, np.float64) - out[:, 0]
    return float(np.mean(0.5 * (s + dy * dy * np.exp(-s))))
