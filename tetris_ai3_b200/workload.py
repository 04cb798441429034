"""Synthetic workloads for the model x game evaluation.

The reference trains on its own seeded games; nothing here is a dataset. The
weight vectors below are drawn from a pinned counter-based generator so every
machine builds the same inputs for the same config:

* ``splitmix_uniform(seed, n)`` -- the i-th value is the splitmix64 output for
  state ``seed + (i+1) * 0x9e3779b97f4a7c15`` (the stream that seeds
  xoshiro256** in ta3_sim/incl/ta3/sim/utility/xoshiro256ss.hpp:20-28), mapped
  to [0, 1) with 53 bits.
* ``normal(seed, n)`` -- Box-Muller in float64 over consecutive uniform pairs.

Game seeds follow the reference: either given directly (the 1-model x 8-game case uses 0..7)
or derived like ``ta3::gpu::simulate`` (ta3_gpu/incl/ta3/gpu/model_eval.hpp:148-151):
xoshiro256**(seed) draws, one per game.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

NUM_PARAMS = 97          # ta3_ai/incl/ta3/ai/models/models/model_v11.hpp:44
# the reference's dense layers widened to 10 -> H -> H -> 1 (utility.hpp:29-46 layout per layer:
# [out][in] weights then [out] biases); the kernels are built for H = 64 and H = 32


def wide_layers(hidden: int = 64):
    return ((10, hidden), (hidden, hidden), (hidden, 1))


def wide_params(hidden: int = 64) -> int:
    return sum(i * o + o for i, o in wide_layers(hidden))


WIDE_LAYERS = wide_layers(64)
NUM_PARAMS_WIDE = wide_params(64)        # 4929
NUM_PARAMS_WIDE32 = wide_params(32)      # 1441
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M64 = (1 << 64) - 1


def splitmix_u64(seed: int, n: int) -> np.ndarray:
    """n consecutive splitmix64 outputs of the stream started at ``seed``."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & _M64) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def splitmix_uniform(seed: int, n: int) -> np.ndarray:
    return (splitmix_u64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def normal(seed: int, n: int) -> np.ndarray:
    """n standard normals (float64), Box-Muller over the splitmix64 stream."""
    m = (n + 1) // 2
    u = splitmix_uniform(seed, 2 * m).reshape(m, 2)
    r = np.sqrt(-2.0 * np.log1p(-u[:, 0]))
    t = 2.0 * np.pi * u[:, 1]
    return np.stack([r * np.cos(t), r * np.sin(t)], axis=1).reshape(-1)[:n]


def xoshiro_seeds(seed: int, games: int) -> np.ndarray:
    """The per-game seeds ``ta3::gpu::simulate`` derives from one seed."""
    s = [0, 0, 0, 0]
    x = seed & _M64
    for k in range(4):
        x = (x + 0x9E3779B97F4A7C15) & _M64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        s[k] = z ^ (z >> 31)
    out = np.empty(games, dtype=np.uint64)
    rotl = lambda v, k: ((v << k) | (v >> (64 - k))) & _M64
    for g in range(games):
        out[g] = (rotl((s[1] * 5) & _M64, 7) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
    return out


def load_champ(path: str) -> np.ndarray:
    """A ``.champ`` file: u64 count then that many little-endian float64
    (ta3_trainer/src/trainer2.cpp:252-265). Returned as float32, the evaluator's type."""
    raw = np.fromfile(path, dtype=np.uint8)
    n = int(np.frombuffer(raw[:8], dtype="<u8")[0])
    return np.frombuffer(raw[8:8 + 8 * n], dtype="<f8").astype(np.float32)


def save_champ(path: str, w) -> None:
    w = np.asarray(w, dtype="<f8")
    with open(path, "wb") as f:
        f.write(np.uint64(w.size).astype("<u8").tobytes())
        f.write(w.tobytes())


CHAMPION_PATH = os.path.join(os.path.dirname(__file__), "data", "v11_16_32_32_score_296.champ")


def champion() -> np.ndarray:
    return load_champ(CHAMPION_PATH)


@dataclasses.dataclass
class Batch:
    """One evaluation batch: ``islands`` groups of ``models_per_island`` weight
    vectors; island i's models all play island i's ``games`` seeds."""
    name: str
    weights: np.ndarray          # (islands * models_per_island, num_params) float32
    seeds: np.ndarray            # (islands, games) uint64
    max_moves: int

    @property
    def islands(self) -> int:
        return int(self.seeds.shape[0])

    @property
    def models(self) -> int:
        return int(self.weights.shape[0])

    @property
    def games(self) -> int:
        return int(self.seeds.shape[1])

    @property
    def sims(self) -> int:
        return self.models * self.games


def single_model_batch() -> Batch:
    """1 v11 model, weights N(0, 0.5^2) from seed 0, games with seeds 0..7, cap 500."""
    w = (0.5 * normal(0, NUM_PARAMS)).astype(np.float32)[None, :]
    return Batch("1 model x 8 games, cap 500", w, np.arange(8, dtype=np.uint64)[None, :], 500)


def generation_batch(islands: int = 4, pop: int = 50, games: int = 50, max_moves: int = 2000, seed: int = 1) -> Batch:
    """One CMA-ES generation: islands x pop candidates x games. Island mean
    m ~ N(0, 0.25) (variance 0.25) from ``seed``; candidates N(m, 0.5^2 I);
    island i plays the ``games`` seeds simulate() derives from seed*1000+i."""
    m = 0.5 * normal(seed, NUM_PARAMS)
    z = normal(seed + 0x51ED, islands * pop * NUM_PARAMS).reshape(islands * pop, NUM_PARAMS)
    w = (m[None, :] + 0.5 * z).astype(np.float32)
    seeds = np.stack([xoshiro_seeds(seed * 1000 + i, games) for i in range(islands)])
    return Batch(f"{islands} islands x {pop} x {games} games = {islands * pop * games} sims, cap {max_moves}",
                 w, seeds, max_moves)


def uneven_batch(models: int = 200, games: int = 100, max_moves: int = 10000, seed: int = 2) -> Batch:
    """Uneven lengths: 10 % of the models are the shipped v11 champion, 90 %
    N(0, 1) weights, order shuffled by ``seed``; one island."""
    n_champ = models // 10
    rnd = normal(seed, (models - n_champ) * NUM_PARAMS).reshape(-1, NUM_PARAMS)
    w = np.concatenate([np.repeat(champion()[None, :], n_champ, axis=0), rnd]).astype(np.float32)
    order = np.argsort(splitmix_u64(seed + 7, models), kind="stable")
    seeds = xoshiro_seeds(seed, games)[None, :]
    return Batch(f"{models} models x {games} games (10% champion), cap {max_moves}", w[order], seeds, max_moves)


def wide_scale(hidden: int = 64) -> np.ndarray:
    """Per-parameter standard deviation of the widened network's initialisation:
    1 / sqrt(fan_in) for weights, 0 for biases."""
    parts = []
    for fan_in, fan_out in wide_layers(hidden):
        parts.append(np.full(fan_in * fan_out, 1.0 / np.sqrt(fan_in)))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts)


def wide_batch(islands: int = 8, pop: int = 100, games: int = 100, max_moves: int = 2000, seed: int = 3,
               hidden: int = 64) -> Batch:
    """The widened evaluator's generation: islands x pop models of the 10 -> hidden ->
    hidden -> 1 network, each an independent N(0, 1/fan_in) initialisation drawn from
    ``seed``; island i plays the ``games`` seeds simulate() derives from seed*1000+i."""
    n = wide_params(hidden)
    z = normal(seed, islands * pop * n).reshape(islands * pop, n)
    sc = wide_scale(hidden)
    w = np.where(sc[None, :] > 0, z * sc[None, :], 0.0).astype(np.float32)   # biases exactly +0
    seeds = np.stack([xoshiro_seeds(seed * 1000 + i, games) for i in range(islands)])
    return Batch(f"widened 10-{hidden}-{hidden}-1: {islands} islands x {pop} x {games} games = "
                 f"{islands * pop * games} sims, cap {max_moves}", w, seeds, max_moves)
