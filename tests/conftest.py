"""Shared fixtures: the oracle library (built from oracle/ta3_oracle.c if
absent), the golden vectors, and the `gpu` marker."""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libta3oracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def f32_from_hex(h: str) -> np.float32:
    return np.frombuffer(bytes.fromhex(h)[::-1], dtype=np.float32)[0]


def weights_from_hex(rows) -> np.ndarray:
    return np.array([[f32_from_hex(h) for h in row] for row in rows], dtype=np.float32)


def load_golden(name: str):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    lib = C.CDLL(ORACLE_SO)
    lib.ta3o_evaluate.restype = C.c_float
    return lib


@pytest.fixture(scope="session")
def oracle():
    return _load_oracle()


@pytest.fixture(scope="session")
def golden_games():
    return load_golden("games")


def oracle_eval(lib, w: np.ndarray, seeds: np.ndarray, max_moves: int, threads: int = 8):
    """Batch through the oracle: model-major (score, pieces, lines, total evals)."""
    w = np.ascontiguousarray(w, dtype=np.float32).reshape(-1, 97)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    n = w.shape[0] * seeds.size
    sc = np.zeros(n, np.float32)
    pc = np.zeros(n, np.uint32)
    lc = np.zeros(n, np.uint32)
    ev = C.c_uint64()
    lib.ta3o_eval_mt(ptr(w), w.shape[0], ptr(seeds), seeds.size, max_moves, threads, ptr(sc), ptr(pc), ptr(lc),
                     C.byref(ev))
    return sc, pc, lc, ev.value


HOST_SO = os.path.join(ROOT, "tetris_ai3_b200", "_lib", "libta3b_host.so")


@pytest.fixture(scope="session")
def host():
    """The C++ host library (CMA-ES + island trainer), built if absent."""
    if not os.path.exists(HOST_SO):
        from tetris_ai3_b200 import build as b
        if not os.path.exists(b.LIB):
            b.build_lib()
        b.build_host()
    from tetris_ai3_b200 import trainer
    return trainer


def oracle_play_keys(lib, w: np.ndarray, seed: int, max_moves: int):
    """One game on the oracle with per-move top-two final keys: (trace bytes, n_moves, keys (n, 2))."""
    w = np.ascontiguousarray(w, dtype=np.float32).reshape(97)
    s, p, l, e, nm = C.c_float(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint32()
    tr = np.zeros(3 * max(max_moves, 1), np.uint8)
    keys = np.zeros((max(max_moves, 1), 2), np.uint64)
    lib.ta3o_play_keys(ptr(w), C.c_uint64(int(seed)), max_moves, C.byref(s), C.byref(p), C.byref(l), C.byref(e),
                       ptr(tr), C.byref(nm), ptr(keys))
    return tr[:3 * nm.value].tobytes(), nm.value, keys[:nm.value]


def first_divergence(trace_a: bytes, trace_b: bytes, keys_a, keys_b):
    """The first move where two traces differ, with each side's top-two margin there, or None.
    A divergence between two bit-exact paths can only come from a value that rounds differently;
    the margin says how close that decision was."""
    from tetris_ai3_b200.evaluator import decode_key, top2_margin
    n = min(len(trace_a), len(trace_b)) // 3
    for m in range(n):
        if trace_a[3 * m:3 * m + 3] != trace_b[3 * m:3 * m + 3]:
            side = lambda k: {"best": decode_key(k[m][0]), "second": decode_key(k[m][1]),
                              "margin": top2_margin(k[m][0], k[m][1])}
            return {"move": m, "a": trace_a[3 * m:3 * m + 3].hex(), "b": trace_b[3 * m:3 * m + 3].hex(),
                    "keys_a": side(keys_a), "keys_b": side(keys_b)}
    if len(trace_a) != len(trace_b):
        return {"move": n, "a": trace_a[3 * n:3 * n + 3].hex(), "b": trace_b[3 * n:3 * n + 3].hex()}
    return None
