"""Pins the oracle (oracle/ta3_oracle.c) to the reference: every golden vector
in tests/golden/ was produced by the reference's own CPU code (gen_golden.py),
and the known-answer facts below restate the reference tests' assertions."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import f32_from_hex, load_golden, ptr, weights_from_hex

PIECES = "IOTSZJL"


def test_placement_counts_kat(oracle):
    # ta3_ai/tests/src/search/search_test.cpp:60-67
    want = {"O": 9, "I": 17, "S": 17, "Z": 17, "T": 34, "J": 34, "L": 34}
    for p, name in enumerate(PIECES):
        buf = [(C.c_uint8 * 40)(), (C.c_int8 * 40)(), (C.c_uint16 * 40)(), (C.c_int8 * 40)()]
        assert oracle.ta3o_placements(p, *buf) == want[name]


def test_placement_lut_matches_reference(oracle):
    g = load_golden("tables")
    for p in range(7):
        buf = [(C.c_uint8 * 40)(), (C.c_int8 * 40)(), (C.c_uint16 * 40)(), (C.c_int8 * 40)()]
        n = oracle.ta3o_placements(p, *buf)
        got = [[buf[0][i], buf[1][i], buf[2][i], buf[3][i]] for i in range(n)]
        assert got == g["placements"][str(p)]


def test_plan_trees_match_reference(oracle):
    g = load_golden("tables")
    for he in (0, 1):
        counts, nodes = (C.c_uint32 * 4)(), (C.c_uint8 * 384)()
        oracle.ta3o_plan_tree(he, counts, nodes)
        nd = np.frombuffer(nodes, np.uint8).reshape(4, 16, 6)
        got = [[nd[l, n].tolist() for n in range(counts[l])] for l in range(4)]
        assert got == g["plan_trees"][str(he)]
    # beam_test.cpp:43-65 consistency: child ranges tile the next layer, parents link back
    for tree in load_golden("tables")["plan_trees"].values():
        for l in range(3):
            nxt = 0
            for n, node in enumerate(tree[l]):
                assert node[2] == nxt and node[3] >= node[2]
                for c in range(node[2], node[3]):
                    assert tree[l + 1][c][1] == n
                nxt = node[3]
            assert nxt == len(tree[l + 1])


def test_search_constants():
    c = load_golden("tables")["consts"]
    assert c == {"DEPTH": 4, "MAX_PLACEMENTS": 34, "MAX_ROOT_GROUPS": 2, "MAX_CHILD_MID": 2, "MAX_LAST": 2,
                 "ROOT_SLOTS": 68, "MID_SLOTS": 2176, "LEAF_ORDERS": 2176, "ORDER_SPAN": 2192}


def test_engine_queues_and_seed_streams(oracle):
    g = load_golden("engine")
    for s, q in g["queues"].items():
        out = (C.c_uint32 * 6)()
        oracle.ta3o_piece_queue(C.c_uint64(int(s)), out)
        assert list(out) == q
    for s, seq in g["simulate_seeds"].items():
        out = np.zeros(16, np.uint64)
        oracle.ta3o_simulate_seeds(C.c_uint64(int(s)), 16, ptr(out))
        assert [str(int(v)) for v in out] == seq


def test_bag_is_a_permutation(oracle):
    # tetris_engine_test.cpp:34-45: every 7 consecutive bag draws are a permutation
    for seed in (7, 42, 2**40 + 3):
        seq = np.zeros(70, np.uint8)
        oracle.ta3o_piece_sequence(C.c_uint64(seed), 70, ptr(seq))
        for k in range(10):
            assert sorted(seq[7 * k:7 * k + 7].tolist()) == list(range(7))


def test_board_primitives_match_reference(oracle):
    g = load_golden("boards")
    for a in g["applies"]:
        cols = np.array(a["cols"], np.uint32)
        out = np.zeros(10, np.uint32)
        cl = C.c_uint32()
        ok = oracle.ta3o_apply(ptr(cols), a["piece"], a["index"], ptr(out), C.byref(cl))
        assert ok == a["legal"]
        if ok:
            assert out.tolist() == a["out"] and cl.value == a["cleared"]


def test_features_and_value_match_reference(oracle):
    g = load_golden("boards")
    w = np.array([f32_from_hex(h) for h in g["weights"]], np.float32)
    for f in g["features"]:
        cols = np.array(f["cols"], np.uint32)
        feats = np.zeros(10, np.float32)
        v = np.float32(oracle.ta3o_evaluate(ptr(w), ptr(cols), C.c_uint32(f["clear_bits"]), f["held_i"], ptr(feats)))
        assert [x.tobytes() for x in feats] == [f32_from_hex(h).tobytes() for h in f["features"]]
        assert v.tobytes() == f32_from_hex(f["value"]).tobytes()


def test_board_metric_kats(oracle):
    # board2_test.cpp:123-133: O pillars in cols 3,4 bridged by an I leave 12 holes under cols 5,6
    cols = np.zeros(10, np.uint32)
    for x in (3, 4):
        cols[x] = sum(1 << y for y in range(17, 23))
    for x in (3, 4, 5, 6):
        cols[x] |= 1 << 16
    out = np.zeros(5, np.uint32)
    oracle.ta3o_board_ints(ptr(cols), ptr(out))
    assert out[0] == 12                       # holes
    assert out[2] == 7                        # max height: row 16 -> 23 - 16
    # board2_test.cpp:97-112: O on an empty board lands with its top at y=21, vertical I at y=19
    empty = np.zeros(10, np.uint32)
    res = np.zeros(10, np.uint32)
    cl = C.c_uint32()
    assert oracle.ta3o_apply(ptr(empty), 1, 4, ptr(res), C.byref(cl)) == 1   # O, x=3
    assert res[4] == res[5] == (1 << 21) | (1 << 22)
    assert oracle.ta3o_apply(ptr(empty), 0, 7, ptr(res), C.byref(cl)) == 1   # I vertical at col 0
    assert res[0] == sum(1 << y for y in range(19, 23))


def _check_case(oracle, case, max_games=None):
    w = weights_from_hex(case["weights"])
    for m, row in enumerate(case["results"]):
        for r in row[:max_games]:
            s, p, l, e, nm = C.c_float(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint32()
            tr = (C.c_uint8 * (3 * case["max_moves"]))()
            bd = np.zeros(10, np.uint32)
            oracle.ta3o_play(ptr(w[m]), C.c_uint64(int(r["seed"])), case["max_moves"], C.byref(s), C.byref(p),
                             C.byref(l), C.byref(e), tr, C.byref(nm), ptr(bd))
            where = f'{case["name"]} model {m} seed {r["seed"]}'
            assert bytes(tr)[:3 * nm.value].hex() == r["trace"], where
            assert np.float32(s.value).tobytes() == f32_from_hex(r["score"]).tobytes(), where
            assert (p.value, l.value, e.value, nm.value) == (r["pieces"], r["lines"], r["evals"], r["moves"]), where
            assert bd.tolist() == r["board"], where


@pytest.mark.parametrize("idx", range(7))
def test_games_match_reference(oracle, golden_games, idx):
    cases = golden_games["cases"]
    if idx >= len(cases):
        pytest.skip("no such case")
    case = cases[idx]
    # the long champion cases are the slowest: sample their games
    limit = 8 if "seeds 0..29" in case["name"] else None
    _check_case(oracle, case, limit)


def test_random_weight_games_match_reference(oracle, golden_games):
    case = [c for c in golden_games["cases"] if c["name"].startswith("random")][0]
    w = weights_from_hex(case["weights"])
    seeds = np.array([int(s) for s in case["seeds"]], np.uint64)
    from conftest import oracle_eval
    sc, pc, lc, _ = oracle_eval(oracle, w, seeds, case["max_moves"])
    flat = [r for row in case["results"] for r in row]
    assert [x.tobytes().hex() for x in sc] == [f32_from_hex(r["score"]).tobytes().hex() for r in flat]
    assert pc.tolist() == [r["pieces"] for r in flat]
    assert lc.tolist() == [r["lines"] for r in flat]


def test_champion_mean_score(oracle, golden_games):
    case = [c for c in golden_games["cases"] if "seeds 0..29" in c["name"]][0]
    scores = np.array([r["score_f"] for r in case["results"][0]])
    assert abs(scores.mean() - 294.0) < 0.5      # consistent with the "296" champion file name
