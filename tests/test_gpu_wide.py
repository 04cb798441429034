"""The widened network (10 -> 64 -> 64 -> 1, 4,929 weights per model) on the
GPU kernel against the reference's own games (tests/golden/wide.json) and
against the oracle on further random models: bit-exact scores, pieces, lines,
evaluated placements and traces."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import f32_from_hex, load_golden, ptr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ev():
    from tetris_ai3_b200 import ModelEvaluator
    return ModelEvaluator(device=0)


def _golden():
    g = load_golden("wide")
    w = np.stack([np.frombuffer(bytes.fromhex(c["weights_hex"]), "<f4") for c in g["cases"]]).astype(np.float32)
    return g, w, np.array([int(s) for s in g["seeds"]], np.uint64)


def test_wide_matches_reference_games(ev):
    g, w, seeds = _golden()
    out = ev.eval_trace(w, w.shape[0], seeds, g["max_moves"])
    for m, case in enumerate(g["cases"]):
        for k, r in enumerate(case["results"]):
            i = m * seeds.size + k
            assert out["score"][i] == f32_from_hex(r["score"]), (m, k)
            assert out["pieces"][i] == r["pieces"] and out["lines"][i] == r["lines"], (m, k)
            assert out["evals"][i] == r["evals"] and out["moves"][i] == r["moves"], (m, k)
            assert bytes(out["trace"][i][:3 * r["moves"]]).hex() == r["trace"], (m, k)
            assert out["board"][i].tolist() == r["board"], (m, k)


def test_wide_random_models_match_oracle(ev, oracle):
    from tetris_ai3_b200 import workload
    b = workload.wide_batch(islands=2, pop=3, games=4, max_moves=150, seed=5)
    sc, pc, lc = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    for isl in range(b.islands):
        w = np.ascontiguousarray(b.weights[isl * 3:(isl + 1) * 3])
        s = np.ascontiguousarray(b.seeds[isl])
        n = w.shape[0] * s.size
        osc, opc, olc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        ev_total = C.c_uint64()
        oracle.ta3o_eval_net_mt(ptr(w), 64, 64, w.shape[0], ptr(s), s.size, b.max_moves, 8, ptr(osc), ptr(opc),
                                ptr(olc), C.byref(ev_total))
        lo, hi = isl * n, (isl + 1) * n
        assert sc[lo:hi].tobytes() == osc.tobytes()
        assert np.array_equal(pc[lo:hi], opc) and np.array_equal(lc[lo:hi], olc)


def test_v11_and_wide_share_a_context(ev):
    from tetris_ai3_b200 import workload
    g, w, seeds = _golden()
    a = ev.eval(w[:2], 2, seeds[:2], 60)
    b1 = workload.single_model_batch()
    v = ev.eval(b1.weights, 1, b1.seeds[0][:2], 60)
    a2 = ev.eval(w[:2], 2, seeds[:2], 60)
    assert a.tobytes() == a2.tobytes() and v.shape == (2,)


def _oracle_net(oracle, w, seeds, max_moves, hidden=64):
    n = w.shape[0] * seeds.size
    osc, opc, olc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    ev_total = C.c_uint64()
    oracle.ta3o_eval_net_mt(ptr(w), hidden, hidden, w.shape[0], ptr(seeds), seeds.size, max_moves, 8, ptr(osc),
                            ptr(opc), ptr(olc), C.byref(ev_total))
    return osc, opc, olc


def _variant_models():
    """Widened models that exercise the kernel's zero-term skipping from both sides:
    heavily sparse hidden layers (negative first-layer biases), exact zero weights,
    and models where skipping is not allowed (a -0 bias; the kernel then runs every term)."""
    from tetris_ai3_b200 import workload
    b = workload.wide_batch(islands=1, pop=6, games=3, max_moves=120, seed=11)
    w = b.weights.copy()
    assert w.shape[1] == workload.NUM_PARAMS_WIDE
    w1, b1, w2, b2 = slice(0, 640), slice(640, 704), slice(704, 4800), slice(4800, 4864)   # [out][in] then biases
    w[0, b1] = -0.75                              # most first-layer units are zero in every lane
    w[1, b1] = np.float32(-0.0)                   # -0 biases: skipping disabled
    w[2, b2] = np.float32(-0.0)
    w[2, b1] = 0.25
    w[3, w2.start:w2.stop:3] = 0.0                # exact zero weights in layer 2
    w[4, w1.start:w1.stop:2] = 0.0                # and in layer 1
    w[5, b1] = np.linspace(-1.0, 1.0, 64, dtype=np.float32)
    return w, np.ascontiguousarray(b.seeds[0]), b.max_moves


def test_wide_zero_skipping_is_exact(ev, oracle):
    w, seeds, cap = _variant_models()
    sc, pc, lc = ev.eval_full(w, w.shape[0], seeds, cap)
    osc, opc, olc = _oracle_net(oracle, w, seeds, cap)
    assert sc.tobytes() == osc.tobytes()
    assert np.array_equal(pc, opc) and np.array_equal(lc, olc)


def test_wide_device_entry_matches_host_entry(ev):
    import torch
    w, seeds, cap = _variant_models()
    host = ev.eval(w, w.shape[0], seeds, cap)
    dev = torch.device("cuda", 0)
    dw = torch.from_numpy(w).to(dev)
    ds = torch.from_numpy(seeds.view(np.int64).reshape(1, -1)).to(dev)
    score = torch.zeros(w.shape[0] * seeds.size, dtype=torch.float32, device=dev)
    ev.eval_device(dw, ds, cap, score)
    torch.cuda.synchronize()
    assert score.cpu().numpy().tobytes() == host.tobytes()


def test_wide_time_budget_flavour(ev):
    """The widened network's budget-checking kernel: a generous budget scores
    the batch exactly like the ordinary kernel; a budget far below the run time
    ends the launch with TA3B_ERR_TIMEOUT and leaves the context usable."""
    from tetris_ai3_b200 import EvaluatorError
    w, seeds, cap = _variant_models()
    ref = ev.eval_full(w, w.shape[0], seeds, cap)
    try:
        ev.set_time_budget(120.0)
        full = ev.eval_full(w, w.shape[0], seeds, cap)
        assert all(x.tobytes() == y.tobytes() for x, y in zip(ref, full))
        ev.set_time_budget(1e-5)
        with pytest.raises(EvaluatorError, match="time budget"):
            ev.eval_full(w, w.shape[0], seeds, 2000)
    finally:
        ev.set_time_budget(0)
    again = ev.eval_full(w, w.shape[0], seeds, cap)
    assert all(x.tobytes() == y.tobytes() for x, y in zip(ref, again))


def test_width32_matches_reference_games(ev):
    """The 10 -> 32 -> 32 -> 1 instantiation against the reference's own games
    (tests/golden/wide32.json): scores, pieces and lines bit-exact."""
    g = load_golden("wide32")
    w = np.stack([np.frombuffer(bytes.fromhex(c["weights_hex"]), "<f4") for c in g["cases"]]).astype(np.float32)
    seeds = np.array([int(x) for x in g["seeds"]], np.uint64)
    sc, pc, lc = ev.eval_full(w, w.shape[0], seeds, g["max_moves"])
    for m, case in enumerate(g["cases"]):
        for k, r in enumerate(case["results"]):
            i = m * seeds.size + k
            assert sc[i] == f32_from_hex(r["score"]) and pc[i] == r["pieces"] and lc[i] == r["lines"], (m, k)


def test_width32_random_and_skipping_models_match_oracle(ev, oracle):
    """Width 32 on further models: random initialisations, heavily sparse hidden
    layers, and -0 biases (zero-term skipping off), against the oracle."""
    from tetris_ai3_b200 import workload
    b = workload.wide_batch(islands=1, pop=6, games=4, max_moves=150, seed=5, hidden=32)
    w = b.weights.copy()
    b1, b2 = slice(320, 352), slice(1376, 1408)         # [out][in] weights then biases, per layer
    w[0, b1] = -0.75
    w[1, b1] = np.float32(-0.0)
    w[2, b2] = np.float32(-0.0)
    w[3, 352:1376:3] = 0.0
    seeds = np.ascontiguousarray(b.seeds[0])
    sc, pc, lc = ev.eval_full(w, w.shape[0], seeds, b.max_moves)
    osc, opc, olc = _oracle_net(oracle, w, seeds, b.max_moves, hidden=32)
    assert sc.tobytes() == osc.tobytes()
    assert np.array_equal(pc, opc) and np.array_equal(lc, olc)


def test_width32_device_entry_matches_host_entry(ev):
    import torch
    from tetris_ai3_b200 import workload
    b = workload.wide_batch(islands=1, pop=3, games=3, max_moves=80, seed=6, hidden=32)
    host = ev.eval(b.weights, b.models, b.seeds[0], b.max_moves)
    dev = torch.device("cuda", 0)
    score = torch.zeros(b.sims, dtype=torch.float32, device=dev)
    ev.eval_device(torch.from_numpy(b.weights).to(dev), torch.from_numpy(b.seeds.view(np.int64)).to(dev),
                   b.max_moves, score)
    torch.cuda.synchronize()
    assert score.cpu().numpy().tobytes() == host.tobytes()
