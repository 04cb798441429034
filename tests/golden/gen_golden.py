"""Generate the golden vectors under tests/golden/ by running the REFERENCE's own
CPU path (oracle/_ref/libta3ref.so, built by ``make -C oracle`` from the
reference sources; see oracle/ref_harness.cpp).

Run from the repository root in a container that has the reference checkout:

    make -C oracle REF=/path/to/tetris_ai3 && python tests/golden/gen_golden.py

Outputs (committed; the tests read only these, never the reference):
  tables.json    placement LUT, plan trees, search constants
  engine.json    fresh-engine queues and simulate() seed streams
  boards.json    board-primitive and value-model known answers on random boards
  games.json     whole games: score / pieces / lines / evaluated placements,
                 the per-move (hold, orientation, x) trace and the final board
  wide.json      whole games of the widened 10 -> 64 -> 64 -> 1 network
                 (``python tests/golden/gen_golden.py wide`` regenerates only it)
  wide32.json    games of the 10 -> 32 -> 32 -> 1 network (``... gen_golden.py wide32``)
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from tetris_ai3_b200 import workload  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libta3ref.so"))
P = 97


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def f32hex(v: float) -> str:
    return np.float32(v).tobytes()[::-1].hex()


def wlist(w):
    return [f32hex(x) for x in np.asarray(w, np.float32)]


def tables():
    consts = (C.c_uint32 * 9)()
    REF.ta3ref_search_consts(consts)
    lut = {}
    for p in range(7):
        o, x, cols, c0 = (C.c_uint8 * 40)(), (C.c_int8 * 40)(), (C.c_uint16 * 40)(), (C.c_int8 * 40)()
        n = REF.ta3ref_placements(p, o, x, cols, c0)
        lut[str(p)] = [[o[i], x[i], cols[i], c0[i]] for i in range(n)]
    trees = {}
    for he in (0, 1):
        counts, nodes = (C.c_uint32 * 4)(), (C.c_uint8 * 384)()
        REF.ta3ref_plan_tree(he, counts, nodes)
        nd = np.frombuffer(nodes, np.uint8).reshape(4, 16, 6)
        trees[str(he)] = [[nd[l, n].tolist() for n in range(counts[l])] for l in range(4)]
    names = ["DEPTH", "MAX_PLACEMENTS", "MAX_ROOT_GROUPS", "MAX_CHILD_MID", "MAX_LAST", "ROOT_SLOTS",
             "MID_SLOTS", "LEAF_ORDERS", "ORDER_SPAN"]
    return {"consts": dict(zip(names, list(consts))), "placements": lut, "plan_trees": trees}


def engine():
    queues = {}
    for s in list(range(32)) + [2**63 + 5, 0xDEADBEEF, 2**64 - 1]:
        q = (C.c_uint32 * 6)()
        REF.ta3ref_piece_queue(C.c_uint64(s), q)
        queues[str(s)] = list(q)
    sims = {}
    for s in (0, 1, 42, 0x3E28DF7B1811145B):
        out = np.zeros(16, np.uint64)
        REF.ta3ref_simulate_seeds(C.c_uint64(s), 16, ptr(out))
        sims[str(s)] = [str(int(v)) for v in out]
    return {"queues": queues, "simulate_seeds": sims}


def random_board(rng, style):
    cols = np.zeros(10, np.uint32)
    for x in range(10):
        if style == "surface":            # solid stacks with a few holes
            h = int(rng.integers(0, 20))
            c = 0
            for y in range(23 - h, 23):
                if rng.random() > 0.15:
                    c |= 1 << y
            cols[x] = c
        elif style == "nearfull":         # rows close to full, for line clears
            c = 0
            for y in range(12, 23):
                c |= 1 << y
            cols[x] = c
        else:                              # arbitrary bits, including the spawn rows
            cols[x] = int(rng.integers(0, 1 << 23)) & int(rng.integers(0, 1 << 23))
    if style == "nearfull":               # punch one gap per row in random columns
        for y in range(12, 23):
            x = int(rng.integers(0, 10))
            cols[x] &= ~np.uint32(1 << y)
    return cols


def boards():
    rng = np.random.default_rng(20261203)
    w = (0.5 * workload.normal(99, P)).astype(np.float32)
    feats, applies = [], []
    for k in range(240):
        style = ["surface", "nearfull", "random"][k % 3]
        cols = random_board(rng, style)
        clear_bits = int(sum(int(rng.integers(0, 3)) << (8 * j) for j in range(4)))
        held_i = int(rng.integers(0, 2))
        f = np.zeros(10, np.float32)
        v = REF.ta3ref_evaluate.__call__  # noqa: F841 (keep the symbol check explicit)
        REF.ta3ref_evaluate.restype = C.c_float
        val = REF.ta3ref_evaluate(ptr(w), ptr(cols), C.c_uint32(clear_bits), held_i, ptr(f))
        feats.append({"cols": cols.tolist(), "clear_bits": clear_bits, "held_i": held_i,
                      "features": wlist(f), "value": f32hex(val)})
        for _ in range(4):
            piece = int(rng.integers(0, 7))
            n = {0: 17, 1: 9, 2: 34, 3: 17, 4: 17, 5: 34, 6: 34}[piece]
            idx = int(rng.integers(0, n))
            out = np.zeros(10, np.uint32)
            cl = C.c_uint32()
            ok = REF.ta3ref_apply(ptr(cols), piece, idx, ptr(out), C.byref(cl))
            applies.append({"cols": cols.tolist(), "piece": piece, "index": idx, "legal": int(ok),
                            "out": out.tolist(), "cleared": cl.value})
    return {"weights": wlist(w), "features": feats, "applies": applies}


def play(w, seed, cap):
    s, p, l, e, nm = C.c_float(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint32()
    tr = (C.c_uint8 * (3 * cap))()
    bd = np.zeros(10, np.uint32)
    REF.ta3ref_play(ptr(w), C.c_uint64(seed), cap, C.byref(s), C.byref(p), C.byref(l), C.byref(e), tr,
                    C.byref(nm), ptr(bd))
    # cross-check the harness loop against ModelEvaluator::eval_host itself
    sd = np.array([seed], np.uint64)
    eh = np.zeros(1, np.float32)
    REF.ta3ref_eval_host(ptr(w), 1, ptr(sd), 1, cap, ptr(eh))
    assert np.float32(eh[0]).tobytes() == np.float32(s.value).tobytes(), (seed, eh[0], s.value)
    return {"seed": str(int(seed)), "max_moves": cap, "score": f32hex(s.value), "score_f": float(s.value),
            "pieces": p.value, "lines": l.value, "evals": e.value, "moves": nm.value,
            "trace": bytes(tr)[:3 * nm.value].hex(), "board": bd.tolist()}


def games():
    cases = []

    def add(name, wmat, seeds, cap):
        wmat = np.asarray(wmat, np.float32).reshape(-1, P)
        res = [[play(wmat[m], int(sd), cap) for sd in seeds] for m in range(wmat.shape[0])]
        cases.append({"name": name, "weights": [wlist(x) for x in wmat], "seeds": [str(int(s)) for s in seeds],
                      "max_moves": cap, "results": res})
        print(name, [[r["pieces"] for r in row] for row in res], flush=True)

    c0 = workload.single_model_batch()
    add("single model: N(0,0.5^2) seed 0, seeds 0..7, cap 500", c0.weights, c0.seeds[0], 500)
    pw = np.zeros(P, np.float32)
    for ms in (11, 22, 33):                                  # parity_test.cpp:51-66
        REF.ta3ref_parity_weights(ms, ptr(pw))
        add(f"parity_test model seed {ms}, seeds 1..4, 200 moves", pw.copy(), [1, 2, 3, 4], 200)
    multi = []
    for ms in (100, 101, 102):                               # parity_test.cpp:70-100
        REF.ta3ref_parity_weights(ms, ptr(pw))
        multi.append(pw.copy())
    add("parity_test multi-model seeds 100..102, seeds 1..4, 200 moves", np.stack(multi), [1, 2, 3, 4], 200)
    sw = np.zeros(2 * P, np.float32)
    REF.ta3ref_selfcheck_weights(ptr(sw))                   # trainer2.cpp:57-89
    add("trainer self-check: 2 models, seeds 101/202/303, 100 moves", sw, [101, 202, 303], 100)
    champ = workload.champion()        # the reference's models/v11_16_32_32_score_296.champ, byte for byte
    add("v11 champion, seeds 0..29, cap 300", champ, list(range(30)), 300)
    add("v11 champion, seed 0, cap 2000", champ, [0], 2000)
    rng = np.random.default_rng(7)
    rw = np.stack([(s * workload.normal(1000 + k, P)) for k, s in enumerate([0.25, 0.5, 1.0, 2.0] * 6)])
    add("random weights x 24 (sigma 0.25..2), 4 seeds, cap 400", rw, [int(x) for x in rng.integers(0, 2**63, 4)], 400)
    return {"cases": cases}


def play_wide(w, seed, cap):
    s, p, l, e, nm = C.c_float(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint32()
    tr = (C.c_uint8 * (3 * cap))()
    bd = np.zeros(10, np.uint32)
    REF.ta3ref_play_wide(ptr(w), C.c_uint64(seed), cap, C.byref(s), C.byref(p), C.byref(l), C.byref(e), tr,
                         C.byref(nm), ptr(bd))
    return {"seed": str(int(seed)), "max_moves": cap, "score": f32hex(s.value), "score_f": float(s.value),
            "pieces": p.value, "lines": l.value, "evals": e.value, "moves": nm.value,
            "trace": bytes(tr)[:3 * nm.value].hex(), "board": bd.tolist()}


def wide():
    """The widened 10 -> 64 -> 64 -> 1 network (the reference's dense layers,
    ta3ref_play_wide): the first models of the widened generation workload
    (N(0, 1/fan_in) from seed 3), its island-0 game seeds, cap 300. Weights are
    stored as little-endian float32 in hex (4,929 per model)."""
    assert REF.ta3ref_num_params_wide() == workload.NUM_PARAMS_WIDE
    b = workload.wide_batch(islands=1, pop=6, games=3, max_moves=300)
    cases = []
    for m in range(b.models):
        w = np.ascontiguousarray(b.weights[m])
        res = [play_wide(w, int(sd), 300) for sd in b.seeds[0]]
        cases.append({"model": m, "weights_hex": w.astype("<f4").tobytes().hex(), "results": res})
        print("wide model", m, [r["pieces"] for r in res], flush=True)
    return {"workload": b.name, "seeds": [str(int(x)) for x in b.seeds[0]], "max_moves": 300, "cases": cases}


def wide32():
    """The same for the 10 -> 32 -> 32 -> 1 network (ta3ref_eval_wide32_mt, one
    thread): per game score, pieces and lines, and the batch's evaluated placements.
    Weights as little-endian float32 hex (1,441 per model)."""
    b = workload.wide_batch(islands=1, pop=6, games=3, max_moves=300, hidden=32)
    seeds = np.ascontiguousarray(b.seeds[0], np.uint64)
    w = np.ascontiguousarray(b.weights, np.float32)
    n = b.models * seeds.size
    sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    ev = C.c_uint64()
    REF.ta3ref_eval_wide32_mt(ptr(w), b.models, ptr(seeds), seeds.size, 300, 1, ptr(sc), ptr(pc), ptr(lc),
                              C.byref(ev))
    cases = []
    for m in range(b.models):
        res = [{"seed": str(int(seeds[g])), "score": f32hex(sc[m * seeds.size + g]),
                "pieces": int(pc[m * seeds.size + g]), "lines": int(lc[m * seeds.size + g])} for g in range(seeds.size)]
        cases.append({"model": m, "weights_hex": w[m].astype("<f4").tobytes().hex(), "results": res})
        print("wide32 model", m, [r["pieces"] for r in res], flush=True)
    return {"workload": b.name, "seeds": [str(int(x)) for x in seeds], "max_moves": 300, "evals_total": ev.value,
            "cases": cases}


def main():
    only = sys.argv[1:]
    for name, fn in (("tables", tables), ("engine", engine), ("boards", boards), ("games", games), ("wide", wide),
                     ("wide32", wide32)):
        if only and name not in only:
            continue
        data = fn()
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(data, f, separators=(",", ":"))
        print("wrote", name)


if __name__ == "__main__":
    main()
