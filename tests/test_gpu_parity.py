"""Parity of the CUDA evaluator (through the C ABI) with the reference:
golden vectors from the reference's own CPU code, the oracle on seeded random
inputs, and size-independent properties at full configuration sizes.
Bit-exact throughout: scores compare as float32 bit patterns."""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import f32_from_hex, first_divergence, oracle_eval, oracle_play_keys, weights_from_hex

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ev():
    from tetris_ai3_b200 import ModelEvaluator
    e = ModelEvaluator(device=0)
    yield e
    e.close()


def _divergence(ev, oracle, w, seed, max_moves):
    """The first move where the device and the oracle part, with both sides' top-two margins."""
    out = ev.eval_trace(w, 1, np.array([seed], np.uint64), max_moves, keys=True)
    nm = int(out["moves"][0])
    otr, _, okeys = oracle_play_keys(oracle, w, seed, max_moves)
    return first_divergence(bytes(out["trace"][0][:3 * nm]), otr, out["keys"][0][:nm], okeys)


def _check_golden_case(ev, case, oracle=None):
    w = weights_from_hex(case["weights"])
    seeds = np.array([int(s) for s in case["seeds"]], np.uint64)
    out = ev.eval_trace(w, w.shape[0], seeds, case["max_moves"])
    flat = [r for row in case["results"] for r in row]
    for i, r in enumerate(flat):
        where = f'{case["name"]} sim {i}'
        nm = int(out["moves"][i])
        if oracle is not None and bytes(out["trace"][i][:3 * nm]).hex() != r["trace"]:
            m, g = divmod(i, seeds.size)
            where += f" divergence {_divergence(ev, oracle, w.reshape(-1, 97)[m], int(seeds[g]), case['max_moves'])}"
        assert bytes(out["trace"][i][:3 * nm]).hex() == r["trace"], where
        assert out["score"][i].tobytes() == f32_from_hex(r["score"]).tobytes(), where
        assert (int(out["pieces"][i]), int(out["lines"][i]), int(out["evals"][i]), nm) == \
               (r["pieces"], r["lines"], r["evals"], r["moves"]), where
        assert out["board"][i].tolist() == r["board"], where


def test_golden_games_bit_exact(ev, golden_games, oracle):
    for case in golden_games["cases"]:
        _check_golden_case(ev, case, oracle)


@pytest.fixture(scope="module")
def ev_solo():
    from tetris_ai3_b200 import ModelEvaluator
    e = ModelEvaluator(device=0)
    e.select_variant(7)                     # the single-warp kernel for every batch size
    yield e
    e.close()


def test_small_batches_run_on_team_kernels(ev, ev_solo):
    """A default context plays a batch of at most 2 games per SM with four warps per game (at most
    4: two), spread one block per SM; a selected variant is kept for every batch. Same bits, same
    evaluation counts."""
    from tetris_ai3_b200 import workload
    b = workload.generation_batch(islands=2, pop=5, games=12, max_moves=300, seed=21)
    out = ev.eval_trace(b.weights[:10], 10, b.seeds[0], b.max_moves)
    info = ev.launch_info()
    assert info["warps_per_block"] == 8 and info["grid"] == min(120, info["sms"])
    ref = ev_solo.eval_trace(b.weights[:10], 10, b.seeds[0], b.max_moves)
    assert ev_solo.launch_info()["warps_per_block"] == 16
    for k in ("score", "pieces", "lines", "evals", "moves", "board"):
        assert out[k].tobytes() == ref[k].tobytes(), k
    for i, nm in enumerate(out["moves"]):                 # a trace row is defined up to its game's moves
        assert out["trace"][i][:3 * nm].tobytes() == ref["trace"][i][:3 * nm].tobytes(), i


def test_tail_handoff_is_bit_identical(ev):
    """A full batch on the default variant hands the games still playing at the launch's tail to
    the paired kernel (checkpointed at a move boundary); every output equals the launch that keeps
    each game on one warp, traces included, and games really were handed over."""
    from tetris_ai3_b200 import workload
    b = workload.generation_batch(islands=4, pop=50, games=50, max_moves=300, seed=3)
    w, seeds = b.weights, b.seeds[0]
    ev.select_variant(7)
    try:
        ev.set_tail_handoff(True)
        on = ev.eval_trace(w, w.shape[0], seeds, b.max_moves)
        handed = ev.handoff_games()
        ev.set_tail_handoff(False)
        off = ev.eval_trace(w, w.shape[0], seeds, b.max_moves)
        assert ev.handoff_games() == 0
    finally:
        ev.set_tail_handoff(True)
    assert 0 < handed <= 4 * ev.launch_info()["sms"]
    for k in ("score", "pieces", "lines", "evals", "moves", "board"):
        assert on[k].tobytes() == off[k].tobytes(), k
    for i, nm in enumerate(on["moves"]):
        assert on["trace"][i][:3 * nm].tobytes() == off["trace"][i][:3 * nm].tobytes(), i
    sc, pc, lc = ev.eval_islands(b.weights, b.seeds, b.max_moves)      # the island entry point hands over too
    assert ev.handoff_games() > 0
    ev.set_tail_handoff(False)
    try:
        s2, p2, l2 = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    finally:
        ev.set_tail_handoff(True)
    assert sc.tobytes() == s2.tobytes() and np.array_equal(pc, p2) and np.array_equal(lc, l2)


def test_team_wait_runs_out_and_the_context_stays_usable():
    """Failure detection without a GPU fault: the test flag makes every team's partners leave at
    launch start, so each leader's first team wait gives up after its 1 s limit; the call reports
    the device status, and the same context then evaluates correctly."""
    import time
    from tetris_ai3_b200 import EvaluatorError, ModelEvaluator, workload
    ev = ModelEvaluator(device=0)           # the default launch policy: a small batch runs on a team kernel
    b = workload.generation_batch(islands=1, pop=2, games=10, max_moves=60, seed=5)
    ref = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    ev.set_test_flags(1)
    try:
        t0 = time.perf_counter()
        with pytest.raises(EvaluatorError, match="status 4"):
            ev.eval_islands(b.weights, b.seeds, b.max_moves)
        waited = time.perf_counter() - t0
    finally:
        ev.set_test_flags(0)
    assert 0.9 < waited < 30
    assert ev.launch_info()["warps_per_block"] == 8               # it ran on a team kernel
    out = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    assert all(x.tobytes() == y.tobytes() for x, y in zip(out, ref))
    assert ev.device_status() == 0
    ev.close()


def test_golden_games_single_warp_kernel(ev_solo, golden_games):
    """The golden batches are small, so a default context plays them on the paired kernel; the
    single-warp kernel plays them bit for bit too."""
    for case in golden_games["cases"]:
        _check_golden_case(ev_solo, case)


def test_trace_keys_match_oracle(ev, oracle, golden_games):
    """Per move, the device's two largest final keys (the tracing flavour) equal the oracle's bit
    for bit, so every decision's top-two margin is the reference algorithm's; the tracing flavour
    plays the same games as the ordinary kernel."""
    from tetris_ai3_b200 import workload
    from tetris_ai3_b200.evaluator import top2_margin
    case = next(c for c in golden_games["cases"] if c["name"].startswith("parity_test multi-model"))
    w = np.concatenate([weights_from_hex(case["weights"]).reshape(-1, 97),
                        np.stack([(s * workload.normal(8100 + k, 97)).astype(np.float32)
                                  for k, s in enumerate([0.3, 1.0, 2.0])])])
    seeds = np.array([int(s) for s in case["seeds"]], np.uint64)
    out = ev.eval_trace(w, w.shape[0], seeds, 200, keys=True)
    plain = ev.eval_trace(w, w.shape[0], seeds, 200)
    assert plain["trace"].tobytes() == out["trace"].tobytes() and plain["score"].tobytes() == out["score"].tobytes()
    margins = []
    for i in range(w.shape[0] * seeds.size):
        m, g = divmod(i, seeds.size)
        nm = int(out["moves"][i])
        otr, onm, okeys = oracle_play_keys(oracle, w[m], int(seeds[g]), 200)
        rep = first_divergence(bytes(out["trace"][i][:3 * nm]), otr, out["keys"][i][:nm], okeys)
        assert rep is None and nm == onm, f"sim {i}: {rep}"
        assert np.array_equal(out["keys"][i][:nm], okeys), f"sim {i}"
        margins += [top2_margin(a, b) for a, b in okeys if b]
    assert min(margins) >= 0.0


def test_single_model_matches_golden(ev, golden_games):
    from tetris_ai3_b200 import workload
    b = workload.single_model_batch()
    case = golden_games["cases"][0]
    assert np.array_equal(weights_from_hex(case["weights"]), b.weights)
    sc, pc, lc = ev.eval_full(b.weights, 1, b.seeds[0], b.max_moves)
    flat = case["results"][0]
    assert [x.tobytes() for x in sc] == [f32_from_hex(r["score"]).tobytes() for r in flat]
    assert pc.tolist() == [r["pieces"] for r in flat]
    assert lc.tolist() == [r["lines"] for r in flat]


def test_batched_equals_per_model(ev):
    # ta3_gpu/tests/src/parity_test.cpp:70-100
    from tetris_ai3_b200 import workload
    w = np.stack([(0.7 * workload.normal(300 + m, 97)).astype(np.float32) for m in range(5)])
    seeds = np.array([1, 2, 3, 4], np.uint64)
    batched = ev.eval_full(w, 5, seeds, 200)
    for m in range(5):
        single = ev.eval_full(w[m], 1, seeds, 200)
        for a, b in zip(batched, single):
            assert a[m * 4:(m + 1) * 4].tobytes() == b.tobytes()


def test_random_models_match_oracle(ev, oracle):
    from tetris_ai3_b200 import workload
    rng = np.random.default_rng(5)
    sig = np.array([0.3, 0.5, 1.0, 1.5] * 12)
    w = np.stack([(s * workload.normal(7000 + k, 97)).astype(np.float32) for k, s in enumerate(sig)])
    seeds = rng.integers(0, 2**63, 6, dtype=np.uint64)
    sc, pc, lc = ev.eval_full(w, w.shape[0], seeds, 150)
    osc, opc, olc, _ = oracle_eval(oracle, w, seeds, 150)
    assert sc.tobytes() == osc.tobytes()
    assert np.array_equal(pc, opc) and np.array_equal(lc, olc)


def test_islands_equal_separate_calls(ev):
    from tetris_ai3_b200 import workload
    b = workload.generation_batch(islands=3, pop=4, games=5, max_moves=120, seed=9)
    sc, pc, lc = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    for i in range(3):
        s2, p2, l2 = ev.eval_full(b.weights[i * 4:(i + 1) * 4], 4, b.seeds[i], b.max_moves)
        assert sc[i * 20:(i + 1) * 20].tobytes() == s2.tobytes()
        assert np.array_equal(pc[i * 20:(i + 1) * 20], p2) and np.array_equal(lc[i * 20:(i + 1) * 20], l2)


def test_edge_cases(ev):
    from tetris_ai3_b200 import EvaluatorError, workload
    w = (0.5 * workload.normal(1, 97)).astype(np.float32)
    # max_moves = 0: no piece placed -> -1e6 (model_eval_host.cpp:51)
    sc, pc, lc = ev.eval_full(w, 1, np.array([3, 4], np.uint64), 0)
    assert sc.tolist() == [-1.0e6, -1.0e6] and pc.tolist() == [0, 0]
    # empty batches
    assert ev.eval_full(w[:0], 0, np.array([1], np.uint64), 10)[0].size == 0
    assert ev.eval_full(w, 1, np.array([], np.uint64), 10)[0].size == 0
    # parameter-count mismatch raises (model_eval.cu:110-111)
    with pytest.raises(EvaluatorError):
        ev.eval(np.zeros(96, np.float32), 1, np.array([1], np.uint64), 5)
    # extreme seeds and a single move
    seeds = np.array([0, 2**64 - 1, 2**63], np.uint64)
    sc, pc, lc = ev.eval_full(w, 1, seeds, 1)
    assert pc.tolist() == [1, 1, 1]


def test_extreme_weights_match_oracle(ev, oracle):
    # all-zero weights (every value ties at +0: tie-breaks decide everything), huge and tiny magnitudes
    from tetris_ai3_b200 import workload
    w = np.stack([np.zeros(97, np.float32),
                  (300.0 * workload.normal(11, 97)).astype(np.float32),
                  (1e-3 * workload.normal(12, 97)).astype(np.float32),
                  np.where(workload.normal(13, 97) > 0, 1.0, -1.0).astype(np.float32)])
    seeds = np.array([5, 6, 7], np.uint64)
    sc, pc, lc = ev.eval_full(w, 4, seeds, 120)
    osc, opc, olc, _ = oracle_eval(oracle, w, seeds, 120)
    assert sc.tobytes() == osc.tobytes() and np.array_equal(pc, opc) and np.array_equal(lc, olc)


def test_full_generation_properties(ev, oracle):
    # the full generation (4 x 50 models x 50 games, cap 2000): deterministic, island-consistent, and a sample matches the oracle
    from tetris_ai3_b200 import workload
    b = workload.generation_batch()
    sc1, pc1, lc1 = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    sc2, pc2, lc2 = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    assert sc1.tobytes() == sc2.tobytes() and np.array_equal(pc1, pc2)
    assert (pc1 <= b.max_moves).all() and (lc1 <= 4 * pc1).all()
    # samples of island 0 replayed by the oracle: the 24 shortest sims (early deaths) and the 16
    # longest (cap-reaching CMA candidates, which carry most of the placements), one host thread each
    order = np.argsort(pc1[:50 * 50], kind="stable")
    idx = np.concatenate([order[:24], order[-16:]])
    assert pc1[order[-16:]].min() >= 1000, "the longest sims of the generation play long games"

    def replay(i):
        m, g = divmod(int(i), 50)
        osc, opc, olc, _ = oracle_eval(oracle, b.weights[m], b.seeds[0][g:g + 1], b.max_moves, threads=1)
        return int(i), osc[0], int(opc[0]), int(olc[0])

    with ThreadPoolExecutor(max_workers=16) as pool:
        for i, osc, opc, olc in pool.map(replay, idx):
            assert (osc.tobytes(), opc, olc) == (sc1[i].tobytes(), int(pc1[i]), int(lc1[i])), f"sim {i}"


def test_device_core_matches_host_core(ev):
    """The per-candidate core on the device (fast and full path, one thread per
    candidate) equals the host build of the same code on random records."""
    import ctypes as C
    from tetris_ai3_b200 import build, library, workload
    from test_core_host import boards, NPLACE
    from conftest import ptr
    host = C.CDLL(build.CORETEST_LIB) if __import__("os").path.exists(build.CORETEST_LIB) else \
        C.CDLL(build.build_coretest())
    rng = np.random.default_rng(3)
    w = (0.5 * workload.normal(77, 97)).astype(np.float32)
    bds = [b for b in boards(rng, 120) if not (int(np.bitwise_and.reduce(b)) & ((1 << 23) - 1))]
    host.ta3bt_rec_words.restype = C.c_uint32
    recs = np.zeros((len(bds), host.ta3bt_rec_words()), np.uint32)
    for k, b in enumerate(bds):
        clears = int(rng.integers(0, 3)) | (int(rng.integers(0, 2)) << 16)
        host.ta3bt_build_record(ptr(b), C.c_uint32(clears), ptr(w), ptr(recs[k]))
    cand = np.array([p | (i << 8) | (int(rng.integers(0, 2)) << 16) | (k << 17)
                     for k in range(len(bds)) for p in range(7) for i in range(NPLACE[p])], np.uint32)
    n = cand.size
    fv, fs, uv, ul = np.zeros(n, np.float32), np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros(n, np.int32)
    dd = np.zeros((n, 32), np.float32)
    assert library().ta3b_core_selftest(ptr(recs), len(bds), ptr(cand), n, ptr(w), ptr(fv), ptr(fs), ptr(uv),
                                        ptr(ul), ptr(dd)) == 0
    hv, hs = C.c_float(), None
    hd = np.zeros(32, np.float32)
    mism = []
    for t in range(n):
        c = int(cand[t])
        p, i, held, k = c & 0xFF, (c >> 8) & 0xFF, (c >> 16) & 1, c >> 17
        hd[:] = 0
        st = host.ta3bt_fast(ptr(recs[k]), p, i, held, ptr(w), C.byref(hv), ptr(hd))
        if st != fs[t] or (st == 0 and np.float32(hv.value).tobytes() != fv[t].tobytes()):
            diff = [j for j in range(18) if hd[j].tobytes() != dd[t][j].tobytes()]
            mism.append(("fast", t, p, i, st, int(fs[t]), hv.value, float(fv[t]), "first differing diag",
                         diff[:3], [float(hd[j]) for j in diff[:3]], [float(dd[t][j]) for j in diff[:3]]))
        v2, cl, out = C.c_float(), C.c_uint32(), np.zeros(10, np.uint32)
        lg = host.ta3bt_full(ptr(recs[k][8:18].copy()), C.c_uint32(int(recs[k][18])), p, i, held, ptr(w),
                             C.byref(v2), C.byref(cl), ptr(out))
        if lg != ul[t] or (lg and np.float32(v2.value).tobytes() != uv[t].tobytes()):
            mism.append(("full", t, p, i, lg, int(ul[t]), v2.value, float(uv[t])))
    for m in mism[:8]:
        print("MISMATCH", m)
    # the MLP arithmetic modes (diagnostic slots 29-31) against the kernel's: the scalar mode is the
    # kernel's; the packed modes are reported (their multiply-add pairs are not the reference's
    # separately rounded operations once compiled, see the kernel's MLP mode notes)
    ok = fs == 0
    bad = {name: int((ok & (dd[:, slot].view(np.uint32) != fv.view(np.uint32))).sum())
           for name, slot in (("packed multiplies", 28), ("scalar", 29), ("packed intrinsics", 30),
                              ("packed PTX", 31))}
    print("MLP mode mismatches:", bad, "of", int(ok.sum()))
    assert not mism, f"{len(mism)} of {n} candidates differ"
    assert bad["scalar"] == 0 and bad["packed multiplies"] == 0, bad


def test_generation_graph_replays_match_direct_calls(ev):
    """The per-generation CUDA graph (pinned H2D, kernel, D2H) gives the direct
    call's results, and replays correctly with new populations."""
    from tetris_ai3_b200 import workload
    from tetris_ai3_b200.evaluator import GenerationGraph
    g = GenerationGraph(ev, models=8, islands=2, games=6, max_moves=140)
    for seed in (31, 32):
        b = workload.generation_batch(islands=2, pop=4, games=6, max_moves=140, seed=seed)
        sc, pc, lc, ec = g.run(b.weights, b.seeds)
        s2, p2, l2 = ev.eval_islands(b.weights, b.seeds, b.max_moves)
        assert sc.tobytes() == s2.tobytes() and np.array_equal(pc, p2) and np.array_equal(lc, l2)
        assert (ec > 0).all()


def test_generation_graph_with_tail_handoff(ev):
    """A full generation captured as a CUDA graph runs both kernels of the tail hand-off (the
    single-warp kernel and the paired kernel) and replays the direct call's results."""
    from tetris_ai3_b200 import workload
    from tetris_ai3_b200.evaluator import GenerationGraph
    g = GenerationGraph(ev, models=200, islands=4, games=50, max_moves=120)
    for seed in (41, 42):
        b = workload.generation_batch(islands=4, pop=50, games=50, max_moves=120, seed=seed)
        sc, pc, lc, ec = g.run(b.weights, b.seeds)
        assert ev.handoff_games() > 0
        s2, p2, l2 = ev.eval_islands(b.weights, b.seeds, b.max_moves)
        assert ev.launch_info()["kernels"] == 2
        assert sc.tobytes() == s2.tobytes() and np.array_equal(pc, p2) and np.array_equal(lc, l2)


def test_device_entry_point_with_the_hand_off_and_no_optional_outputs(ev):
    """ta3b_eval_device on a full batch (tail hand-off) with only the score buffer: the handed-over
    games carry no evaluation count, and the scores equal the host entry point's."""
    import torch
    from tetris_ai3_b200 import workload
    b = workload.generation_batch(islands=4, pop=50, games=50, max_moves=120, seed=44)
    w = torch.from_numpy(b.weights).cuda()
    s = torch.from_numpy(b.seeds.view(np.int64)).cuda()
    score = torch.empty(w.shape[0] * b.seeds.shape[1], dtype=torch.float32, device="cuda")
    ev.eval_device(w, s, b.max_moves, score, num_islands=4)
    torch.cuda.synchronize()
    assert ev.device_status() == 0 and ev.launch_info()["kernels"] == 2 and ev.handoff_games() > 0
    sc, _, _ = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    assert score.cpu().numpy().tobytes() == sc.tobytes()


def test_time_budget_stops_the_launch_and_keeps_the_context(ev):
    """A budget far below the batch's run time ends the launch early with
    TA3B_ERR_TIMEOUT (no fault); without a budget the same context then scores
    the batch exactly as before."""
    from tetris_ai3_b200 import EvaluatorError, workload
    b = workload.generation_batch(islands=2, pop=20, games=20, max_moves=2000, seed=3)
    ref = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    ev.set_time_budget(1e-4)
    with pytest.raises(EvaluatorError, match="time budget"):
        ev.eval_islands(b.weights, b.seeds, b.max_moves)
    ev.set_time_budget(0)
    again = ev.eval_islands(b.weights, b.seeds, b.max_moves)
    assert all(x.tobytes() == y.tobytes() for x, y in zip(ref, again))
    with pytest.raises(EvaluatorError):
        ev.set_time_budget(-1.0)

