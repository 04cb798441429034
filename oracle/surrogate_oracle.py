"""CPU checker for the surrogate MLP kernels (tetris_ai3_b200/csrc/ta3s_surrogate.cu).

Test infrastructure only: imported by tests/, never by the product. The
surrogate has no counterpart in the reference, so this is a plain restatement
of the model the kernels compute -- 97 -> 128 -> 128 -> 2, ReLU, Gaussian NLL
0.5 * (s + (y - mu)^2 exp(-s)) averaged over the batch -- in float64, with
every tensor-core operand rounded to BF16 (round to nearest even) exactly
where the kernels round it:
  X, W1, W2, relu(H1), relu(H2) (for dW3), [valid, dmu, ds] (for dW3, db1, db2),
  dH2, dH1 (masked).
The output layer, the loss and dH2 before rounding use FP32-exact inputs
(W3, biases, relu(H2) in full precision), as the kernels do on the CUDA cores.
Parameter layout: W1 [128][112] (columns 97.. zero), W2 [128][128], W3 [2][128],
b1, b2 [128], b3 [2].
"""
from __future__ import annotations

import numpy as np

IN, IN_K, HID = 97, 112, 128
OFF_W1 = 0
OFF_W2 = OFF_W1 + HID * IN_K
OFF_W3 = OFF_W2 + HID * HID
OFF_B1 = OFF_W3 + 2 * HID
OFF_B2 = OFF_B1 + HID
OFF_B3 = OFF_B2 + HID
NPARAM = OFF_B3 + 2


def _bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    w1 = p[OFF_W1:OFF_W2].reshape(HID, IN_K)[:, :IN]
    w2 = p[OFF_W2:OFF_W3].reshape(HID, HID)
    w3 = p[OFF_W3:OFF_B1].reshape(2, HID)
    return w1, w2, w3, p[OFF_B1:OFF_B2], p[OFF_B2:OFF_B3], p[OFF_B3:NPARAM]


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    w1 = rng.uniform(-1, 1, (HID, IN)) * np.sqrt(6 / IN)
    p[OFF_W1:OFF_W2].reshape(HID, IN_K)[:, :IN] = w1
    p[OFF_W2:OFF_W3] = (rng.uniform(-1, 1, HID * HID) * np.sqrt(6 / HID))
    p[OFF_W3:OFF_B1] = rng.uniform(-1, 1, 2 * HID) * np.sqrt(1 / HID)
    p[OFF_B1:OFF_B3] = rng.uniform(-0.1, 0.1, 2 * HID)
    p[OFF_B3:] = rng.uniform(-0.1, 0.1, 2)
    return p


def _exact(a):
    return np.asarray(a, dtype=np.float64)


def forward(p: np.ndarray, x: np.ndarray, rounded: bool = True):
    """(mean, log-variance) per row, and the intermediates the backward pass needs.
    rounded=False drops every BF16 / FP32 rounding (for finite-difference checks)."""
    bf16 = _bf16 if rounded else _exact
    p = np.asarray(p, np.float32 if rounded else np.float64)
    w1, w2, w3, b1, b2, b3 = (np.asarray(t, np.float64) for t in unpack(p))
    xb = bf16(x)
    h1 = np.maximum(xb @ bf16(w1).T + b1, 0.0)
    h1b = bf16(h1)
    z2 = h1b @ bf16(w2).T + b2
    h2 = np.maximum(z2, 0.0)
    h2f = h2.astype(np.float32).astype(np.float64) if rounded else h2
    out = h2f @ w3.T + b3
    return out, dict(xb=xb, h1b=h1b, z2=z2, h2f=h2f, w2=w2, w3=w3)


def gradients(p: np.ndarray, x: np.ndarray, y: np.ndarray, rounded: bool = True):
    """Gradient of the mean NLL (parameter layout) and the summed loss."""
    bf16 = _bf16 if rounded else _exact
    f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if rounded else _exact
    out, c = forward(p, x, rounded)
    n = len(x)
    mu, s_raw = out[:, 0], out[:, 1]
    s = np.clip(s_raw, -12.0, 12.0)
    e = np.exp(-s)
    d = np.asarray(y, np.float64) - mu
    loss = float(np.sum(0.5 * (s + d * d * e)))
    dmu = f32(-d * e / n)
    ds = f32(np.where((s_raw > -12) & (s_raw < 12), 0.5 * (1 - d * d * e) / n, 0.0))
    g = np.zeros(NPARAM, np.float64)
    gb = np.stack([np.ones(n), bf16(dmu), bf16(ds)], 1)           # the [valid, dmu, ds] tile
    g[OFF_W3:OFF_B1] = (bf16(c["h2f"]).T @ gb[:, 1:3]).T.reshape(-1)
    g[OFF_B3] = dmu.sum()
    g[OFF_B3 + 1] = ds.sum()
    dh2 = np.where(c["z2"] > 0, dmu[:, None] * c["w3"][0] + ds[:, None] * c["w3"][1], 0.0)
    dh2b = bf16(dh2)
    g[OFF_B2:OFF_B3] = dh2b.sum(0)
    g[OFF_W2:OFF_W3] = (dh2b.T @ c["h1b"]).reshape(-1)
    dh1 = np.where(c["h1b"] > 0, dh2b @ bf16(c["w2"]), 0.0)
    dh1b = bf16(dh1)
    g[OFF_B1:OFF_B2] = dh1b.sum(0)
    gw1 = np.zeros((HID, IN_K))
    gw1[:, :IN] = dh1b.T @ c["xb"]
    g[OFF_W1:OFF_W2] = gw1.reshape(-1)
    return g, loss


bf16 = _bf16


def loss_of(p: np.ndarray, x: np.ndarray, y: np.ndarray, rounded: bool = False) -> float:
    """Mean NLL (for finite differences)."""
    out, _ = forward(p, x, rounded)
    s = np.clip(out[:, 1], -12.0, 12.0)
    d = np.asarray(y, np.float64) - out[:, 0]
    return float(np.mean(0.5 * (s + d * d * np.exp(-s))))


def spearman(a, b) -> float:
    ra = np.argsort(np.argsort(a, kind="stable"), kind="stable").astype(np.float64)
    rb = np.argsort(np.argsort(b, kind="stable"), kind="stable").astype(np.float64)
    ra -= ra.mean()
    rb -= rb.mean()
    return float((ra * rb).sum() / np.sqrt((ra * ra).sum() * (rb * rb).sum()))
