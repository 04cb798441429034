"""The kernel's candidate-evaluation core (tetris_ai3_b200/csrc/eval_core.h),
compiled for the host, against the oracle: the full path must equal the
reference algorithm on every (board, placement), and the incremental fast path
must equal the full path wherever it does not defer (no clear, no spawn-area
contact), and must not defer otherwise-plain drops."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, f32_from_hex, load_golden, ptr

NPLACE = [17, 9, 34, 17, 17, 34, 34]


@pytest.fixture(scope="module")
def core():
    from tetris_ai3_b200 import build
    so = build.CORETEST_LIB
    if not os.path.exists(so) or os.path.getmtime(so) < max(
            os.path.getmtime(os.path.join(build.CSRC, f)) for f in ("eval_core.h", "tables.h", "core_selftest.cpp")):
        build.build_coretest()
    return C.CDLL(so)


def boards(rng, n):
    out = []
    g = load_golden("boards")
    for f in g["features"][:60]:
        out.append(np.array(f["cols"], np.uint32))
    for r in load_golden("games")["cases"]:
        for row in r["results"]:
            for res in row[:3]:
                out.append(np.array(res["board"], np.uint32))
    while len(out) < n:
        cols = np.zeros(10, np.uint32)
        style = rng.integers(0, 3)
        for x in range(10):
            h = int(rng.integers(0, 23 if style == 2 else 18))
            c = 0
            for y in range(23 - h, 23):
                if rng.random() > (0.08 if style == 1 else 0.25):
                    c |= 1 << y
            cols[x] = c
        # remove full rows the random fill may have produced (a parent is always cleared)
        full = np.bitwise_and.reduce(cols) & ((1 << 23) - 1)
        if full:
            x = int(rng.integers(0, 10))
            cols[x] &= ~np.uint32(full)
        out.append(cols)
    return out


def test_full_and_fast_paths_match_oracle(core, oracle):
    rng = np.random.default_rng(11)
    from tetris_ai3_b200 import workload
    ws = [(s * workload.normal(500 + k, 97)).astype(np.float32) for k, s in enumerate([0.5, 2.0, 40.0])]
    rec = np.zeros(core.ta3bt_rec_words(), np.uint32)
    out = np.zeros(10, np.uint32)
    feats = np.zeros(10, np.float32)
    n_fast = n_defer = n_legal = 0
    for bi, b in enumerate(boards(rng, 300)):
        full = int(np.bitwise_and.reduce(b)) & ((1 << 23) - 1)
        if full:
            continue                              # not a reachable parent
        w = ws[bi % 3]
        clears = int(rng.integers(0, 3)) | (int(rng.integers(0, 2)) << 8) | (int(rng.integers(0, 2)) << 24)
        core.ta3bt_build_record(ptr(b), C.c_uint32(clears), ptr(w), ptr(rec))
        h = [23 - (int(c).bit_length() and (23 - (int(c) & -int(c)).bit_length() + 1)) for c in b]
        for p in range(7):
            for i in range(NPLACE[p]):
                held = int(rng.integers(0, 2))
                v_full, cl = C.c_float(), C.c_uint32()
                legal = core.ta3bt_full(ptr(b), C.c_uint32(clears), p, i, held, ptr(w), C.byref(v_full),
                                        C.byref(cl), ptr(out))
                # oracle: same legality / board / clear count, and the same value bits
                o_out = np.zeros(10, np.uint32)
                o_cl = C.c_uint32()
                o_legal = oracle.ta3o_apply(ptr(b), p, i, ptr(o_out), C.byref(o_cl))
                assert legal == o_legal
                v_fast = C.c_float()
                st = core.ta3bt_fast(ptr(rec), p, i, held, ptr(w), C.byref(v_fast), None)
                if not legal:
                    assert st == 1
                    continue
                n_legal += 1
                assert out.tolist() == o_out.tolist() and cl.value == o_cl.value
                bump = 0 if cl.value == 0 else 1 << (8 * (cl.value - 1))
                ov = np.float32(oracle.ta3o_evaluate(ptr(w), ptr(out), C.c_uint32(clears + bump), held, ptr(feats)))
                assert np.float32(v_full.value).tobytes() == ov.tobytes()
                if st == 0:
                    n_fast += 1
                    assert cl.value == 0
                    assert np.float32(v_fast.value).tobytes() == ov.tobytes()
                else:
                    n_defer += 1
    assert n_fast > 20000 and n_legal > n_fast
    print("fast", n_fast, "deferred legal", n_defer)


def test_fast_path_does_not_defer_plain_drops(core):
    # empty board, no piece reaches a row, nothing clears: every placement is fast
    w = np.ones(97, np.float32)
    rec = np.zeros(core.ta3bt_rec_words(), np.uint32)
    core.ta3bt_build_record(ptr(np.zeros(10, np.uint32)), C.c_uint32(0), ptr(w), ptr(rec))
    v = C.c_float()
    for p in range(7):
        for i in range(NPLACE[p]):
            assert core.ta3bt_fast(ptr(rec), p, i, 0, ptr(w), C.byref(v), None) == 0
