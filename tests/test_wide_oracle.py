"""The oracle's widened-network restatement (oracle/ta3_oracle.c, dense layers
10 -> 64 -> 64 -> 1 over the v11 inputs) against the reference's own CPU
search with the reference's own dense layers (tests/golden/wide.json, made by
oracle/ref_harness.cpp ta3ref_play_wide): every game's score, pieces, lines,
evaluated placements and per-move trace. No GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import f32_from_hex, load_golden, ptr


@pytest.fixture(scope="module")
def wide():
    return load_golden("wide")


def test_workload_reproduces_the_golden_weights(wide):
    from tetris_ai3_b200 import workload
    b = workload.wide_batch(islands=1, pop=len(wide["cases"]), games=3, max_moves=300)
    assert [str(int(x)) for x in b.seeds[0]] == wide["seeds"]
    for case in wide["cases"]:
        w = np.frombuffer(bytes.fromhex(case["weights_hex"]), "<f4")
        assert w.size == workload.NUM_PARAMS_WIDE and np.array_equal(w, b.weights[case["model"]])


def test_oracle_matches_reference_wide_games(oracle, wide):
    assert oracle.ta3o_net_params(64, 64) == 4929
    seeds = np.array([int(s) for s in wide["seeds"]], np.uint64)
    w = np.stack([np.frombuffer(bytes.fromhex(c["weights_hex"]), "<f4") for c in wide["cases"]]).astype(np.float32)
    n = w.shape[0] * seeds.size
    sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    ev = C.c_uint64()
    assert oracle.ta3o_eval_net_mt(ptr(w), 64, 64, w.shape[0], ptr(seeds), seeds.size, wide["max_moves"], 8, ptr(sc),
                                   ptr(pc), ptr(lc), C.byref(ev)) == 0
    total = 0
    for m, case in enumerate(wide["cases"]):
        for g, r in enumerate(case["results"]):
            i = m * seeds.size + g
            assert sc[i] == f32_from_hex(r["score"]), (m, g)
            assert pc[i] == r["pieces"] and lc[i] == r["lines"], (m, g)
            total += r["evals"]
    assert ev.value == total


def test_oracle_wide_trace_matches_reference(oracle, wide):
    case = wide["cases"][1]                       # a short game: its full trace
    r = case["results"][0]
    w = np.frombuffer(bytes.fromhex(case["weights_hex"]), "<f4").astype(np.float32)
    s, p, l, e, nm = C.c_float(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint32()
    tr = (C.c_uint8 * (3 * 300))()
    bd = np.zeros(10, np.uint32)
    oracle.ta3o_play_net(ptr(w), 64, 64, C.c_uint64(int(r["seed"])), 300, C.byref(s), C.byref(p), C.byref(l),
                         C.byref(e), tr, C.byref(nm), ptr(bd))
    assert nm.value == r["moves"] and bytes(tr)[:3 * nm.value].hex() == r["trace"] and bd.tolist() == r["board"]
    assert e.value == r["evals"]


def test_oracle_matches_reference_width32_games(oracle):
    """The 10 -> 32 -> 32 -> 1 network (tests/golden/wide32.json, made by the
    reference harness's ta3ref_eval_wide32_mt): scores, pieces, lines, placements."""
    from tetris_ai3_b200 import workload
    g = load_golden("wide32")
    assert oracle.ta3o_net_params(32, 32) == workload.NUM_PARAMS_WIDE32 == 1441
    b = workload.wide_batch(islands=1, pop=len(g["cases"]), games=3, max_moves=300, hidden=32)
    seeds = np.array([int(s) for s in g["seeds"]], np.uint64)
    assert np.array_equal(seeds, b.seeds[0])
    w = np.stack([np.frombuffer(bytes.fromhex(c["weights_hex"]), "<f4") for c in g["cases"]]).astype(np.float32)
    assert np.array_equal(w, b.weights)
    n = w.shape[0] * seeds.size
    sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    ev = C.c_uint64()
    assert oracle.ta3o_eval_net_mt(ptr(w), 32, 32, w.shape[0], ptr(seeds), seeds.size, g["max_moves"], 8, ptr(sc),
                                   ptr(pc), ptr(lc), C.byref(ev)) == 0
    for m, case in enumerate(g["cases"]):
        for k, r in enumerate(case["results"]):
            i = m * seeds.size + k
            assert sc[i] == f32_from_hex(r["score"]) and pc[i] == r["pieces"] and lc[i] == r["lines"], (m, k)
    assert ev.value == g["evals_total"]
