"""Decoding the final-argmax keys that ta3b_eval_trace records per move (and the oracle's
ta3o_play_keys), and the divergence report built on them (CPU; the device side is compared
with the oracle in the GPU parity tests).

A key is (ordered_bits(value) << 32) | (ORDER_SPAN - order) (ta3_ai/incl/ta3/ai/search/
beam.hpp:204-224): ordered_bits is a monotone map of float bits, so comparing keys compares
values first and, on ties, prefers the lowest order."""
from __future__ import annotations

import numpy as np

from conftest import first_divergence, load_golden, oracle_play_keys, weights_from_hex


def test_ordered_bits_round_trip_and_order():
    from tetris_ai3_b200.evaluator import ordered_bits, ordered_bits_inv
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.normal(0, 1e3, 2000), rng.normal(0, 1e-3, 2000),
                           [0.0, -0.0, np.inf, -np.inf, 1e-45, -1e-45, 3.4e38, -3.4e38]]).astype(np.float32)
    for v in vals:
        assert ordered_bits_inv(ordered_bits(v)).tobytes() == np.float32(v).tobytes()
    srt = np.sort(vals[np.isfinite(vals) & (vals != 0)])
    codes = [ordered_bits(v) for v in srt]
    assert all(a <= b for a, b in zip(codes, codes[1:]))
    assert ordered_bits(np.float32(-0.0)) < ordered_bits(np.float32(0.0))      # -0 below +0, as in the reference


def test_key_decoding_and_margin():
    from tetris_ai3_b200.evaluator import ORDER_SPAN, decode_key, ordered_bits, top2_margin
    k1 = (ordered_bits(np.float32(2.5)) << 32) | (ORDER_SPAN - 7)
    k2 = (ordered_bits(np.float32(2.25)) << 32) | (ORDER_SPAN - 3)
    v, o = decode_key(k1)
    assert v == np.float32(2.5) and o == 7
    assert top2_margin(k1, k2) == 0.25
    assert decode_key(0) == (None, None) and top2_margin(k1, 0) is None
    # equal values: the lower order has the larger key
    k3 = (ordered_bits(np.float32(2.5)) << 32) | (ORDER_SPAN - 9)
    assert k1 > k3 and top2_margin(k1, k3) == 0.0


def test_oracle_keys_are_consistent_with_its_trace(oracle):
    """On the reference's own games (golden traces), the oracle's per-move keys are ordered
    (best > second), and its chosen moves replay the golden trace."""
    case = next(c for c in load_golden("games")["cases"] if c["name"].startswith("parity_test model seed 11"))
    w = weights_from_hex(case["weights"]).reshape(-1, 97)[0]
    for g, seed in enumerate(case["seeds"][:2]):
        trace, n, keys = oracle_play_keys(oracle, w, int(seed), case["max_moves"])
        assert trace.hex() == case["results"][0][g]["trace"]
        assert n == case["results"][0][g]["moves"] and keys.shape == (n, 2)
        assert (keys[:, 0] > keys[:, 1]).all()
        assert (keys[:, 0] >> np.uint64(32) > 0).all()


def test_divergence_report_on_a_planted_mistake(oracle):
    """A mistake planted in a copy of the oracle's trace is reported at its move, with the
    top-two margin of both sides."""
    from tetris_ai3_b200.evaluator import top2_margin
    case = load_golden("games")["cases"][0]
    w = weights_from_hex(case["weights"]).reshape(-1, 97)[0]
    trace, n, keys = oracle_play_keys(oracle, w, int(case["seeds"][0]), case["max_moves"])
    assert first_divergence(trace, trace, keys, keys) is None
    bad = bytearray(trace)
    m = min(5, n - 1)
    bad[3 * m + 2] ^= 1                                  # another column at move m
    rep = first_divergence(trace, bytes(bad), keys, keys)
    assert rep["move"] == m
    assert rep["keys_a"]["margin"] == top2_margin(keys[m][0], keys[m][1]) and rep["keys_a"]["margin"] >= 0
    assert rep["keys_a"]["best"][0] >= rep["keys_a"]["second"][0]
