"""Python host mirror of the reference evaluator seam, over the C ABI in
include/ta3b.h (tetris_ai3_b200/_lib/libta3b.so).

``ModelEvaluator`` mirrors ``ta3::gpu::ModelEvaluator``
(ta3_gpu/incl/ta3/gpu/model_eval.hpp:27-77) and ``simulate`` mirrors
``ta3::gpu::simulate`` (model_eval.hpp:84-114): same argument meaning,
model-major outputs, and a raised exception where the reference throws
``std::runtime_error``. There is no CPU fallback: without the CUDA library or
a B200 the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .workload import NUM_PARAMS, NUM_PARAMS_WIDE, NUM_PARAMS_WIDE32

# v11 (10 -> 8 -> 1), widened (10 -> 64 -> 64 -> 1, 10 -> 32 -> 32 -> 1)
MODEL_SIZES = (NUM_PARAMS, NUM_PARAMS_WIDE, NUM_PARAMS_WIDE32)


def _rows(weights) -> np.ndarray:
    """Weights as (models, params): a 2-D array keeps its shape, anything else is v11 rows."""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    return w if w.ndim == 2 and w.shape[1] in MODEL_SIZES else w.reshape(-1, NUM_PARAMS)

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libta3b.so")
# TA3B_LIBRARY may name another build of the same C ABI (e.g. an experimental one)
_lib = None

EXPORTS = ["ta3b_create", "ta3b_destroy", "ta3b_last_error", "ta3b_eval", "ta3b_eval_islands", "ta3b_eval_device",
           "ta3b_eval_trace", "ta3b_eval_timed", "ta3b_simulate_seeds", "ta3b_launch_info", "ta3b_num_variants", "ta3b_variant_info",
           "ta3b_variant_warps_per_game", "ta3b_set_tail_handoff", "ta3b_handoff_info",
           "ta3b_set_test_flags",
           "ta3b_select_variant", "ta3b_core_selftest", "ta3b_eval_device_noalloc", "ta3b_set_time_budget",
           "ta3b_device_status", "ta3b_noalloc_status"]


class EvaluatorError(RuntimeError):
    """A failed evaluator call (the reference raises std::runtime_error)."""


class _Config(C.Structure):
    _fields_ = [("device", C.c_int), ("warps_per_block", C.c_uint32), ("blocks_per_sm", C.c_uint32)]


def library(path: str | None = None) -> C.CDLL:
    """Load the C-ABI library; raises if it was not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("TA3B_LIBRARY") or _LIB_PATH
    if not os.path.exists(p):
        raise EvaluatorError(f"CUDA evaluator library missing: {p} (run python -m tetris_ai3_b200.build)")
    lib = C.CDLL(p)
    vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
    lib.ta3b_create.restype = vp
    lib.ta3b_create.argtypes = [C.POINTER(_Config)]
    lib.ta3b_destroy.argtypes = [vp]
    lib.ta3b_last_error.restype = C.c_char_p
    lib.ta3b_last_error.argtypes = [vp]
    lib.ta3b_eval.argtypes = [vp, vp, u32, u32, vp, u32, u32, vp, vp, vp]
    lib.ta3b_eval_islands.argtypes = [vp, vp, u32, u32, u32, vp, u32, u32, vp, vp, vp]
    lib.ta3b_eval_device.argtypes = [vp, vp, u32, u32, u32, vp, u32, u32, vp, vp, vp, vp, vp]
    lib.ta3b_eval_trace.argtypes = [vp, vp, u32, u32, vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.ta3b_eval_timed.argtypes = [vp, vp, u32, u32, u32, vp, u32, u32, vp, vp, vp, vp]
    lib.ta3b_simulate_seeds.argtypes = [u64, u32, vp]
    lib.ta3b_launch_info.argtypes = [vp, vp, vp, vp, vp]
    lib.ta3b_num_variants.argtypes = []
    lib.ta3b_variant_info.argtypes = [C.c_int, vp, vp]
    lib.ta3b_variant_warps_per_game.argtypes = [C.c_int]
    lib.ta3b_set_tail_handoff.argtypes = [vp, C.c_int]
    lib.ta3b_handoff_info.argtypes = [vp, vp]
    lib.ta3b_set_test_flags.argtypes = [vp, u32]
    lib.ta3b_select_variant.argtypes = [vp, C.c_int]
    lib.ta3b_set_time_budget.argtypes = [vp, C.c_double]
    lib.ta3b_core_selftest.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp, vp]
    lib.ta3b_eval_device_noalloc.argtypes = [vp, u32, u32, u32, vp, u32, u32, vp, vp, vp, vp, vp,
                                             C.POINTER(C.c_char_p)]
    lib.ta3b_noalloc_status.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_char_p)]
    lib.ta3b_device_status.argtypes = [vp, C.POINTER(C.c_uint32)]
    if path is None:
        _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def simulate_seeds(seed: int, games: int) -> np.ndarray:
    out = np.zeros(games, np.uint64)
    rc = library().ta3b_simulate_seeds(C.c_uint64(seed & (2**64 - 1)), games, _p(out))
    if rc:
        raise EvaluatorError("ta3b_simulate_seeds failed")
    return out


# The final argmax of a move compares 64-bit keys (ta3_ai/incl/ta3/ai/search/beam.hpp:204-224):
# high word = ordered_bits(value), a monotone map of the float's bits; low word = ORDER_SPAN - order,
# so on equal values the lowest order wins. order < LEAF_ORDERS is a leaf (parent rank * 2 + child
# list) * MAX_PLACEMENTS + placement; LEAF_ORDERS + rank is a frontier node with no child.
ORDER_SPAN = 32 * 2 * 34 + 16
LEAF_ORDERS = 32 * 2 * 34


def ordered_bits_inv(s: int) -> np.float32:
    """The float a key's high word encodes (beam.hpp:209-211)."""
    s = int(s) & 0xFFFFFFFF
    u = (s ^ 0x80000000) if s & 0x80000000 else (~s & 0xFFFFFFFF)
    return np.array([u], np.uint32).view(np.float32)[0]


def ordered_bits(v) -> int:
    """beam.hpp:204-207: the monotone map of a float's bits."""
    u = int(np.array([v], np.float32).view(np.uint32)[0])
    return (~u & 0xFFFFFFFF) if u & 0x80000000 else (u | 0x80000000)


def decode_key(key: int):
    """(value, order) of a final-argmax key; (None, None) for the empty key 0."""
    key = int(key)
    if key == 0:
        return None, None
    return ordered_bits_inv(key >> 32), ORDER_SPAN - (key & 0xFFFFFFFF)


def top2_margin(key1: int, key2: int):
    """How far the chosen key's value lies above the runner-up's (float64 difference of the two
    float32 values); None when the move had a single candidate."""
    v1, _ = decode_key(key1)
    v2, _ = decode_key(key2)
    if v1 is None or v2 is None:
        return None
    return float(np.float64(v1) - np.float64(v2))


class ModelEvaluator:
    """One evaluation context: a CUDA stream plus grow-only device buffers.
    Not thread-safe; use one instance per host thread."""

    def __init__(self, device: int = 0, warps_per_block: int = 0, blocks_per_sm: int = 0):
        self._lib = library()
        cfg = _Config(device, warps_per_block, blocks_per_sm)
        self._ctx = self._lib.ta3b_create(C.byref(cfg))
        if not self._ctx:
            raise EvaluatorError(self._lib.ta3b_last_error(None).decode())

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.ta3b_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise EvaluatorError(self._lib.ta3b_last_error(self._ctx).decode())

    @staticmethod
    def _prep(weights, num_models, seeds):
        w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        s = np.ascontiguousarray(seeds, dtype=np.uint64).reshape(-1)
        if num_models == 0:
            if w.size:
                raise EvaluatorError("weights given for zero models")
        elif w.size % num_models or w.size // num_models not in MODEL_SIZES:
            raise EvaluatorError("weights.size() must equal num_models * NUM_PARAMS (97 or 4929)")
        return w, s

    @staticmethod
    def _nparams(w, num_models) -> int:
        return w.size // num_models if num_models else NUM_PARAMS

    def eval(self, weights, num_models: int, seeds, max_moves: int) -> np.ndarray:
        """Per-(model, game) fitness, model-major (index m * len(seeds) + g)."""
        return self.eval_full(weights, num_models, seeds, max_moves)[0]

    def eval_full(self, weights, num_models: int, seeds, max_moves: int):
        """(score, pieces, lines), each model-major."""
        w, s = self._prep(weights, num_models, seeds)
        n = num_models * s.size
        sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        self._check(self._lib.ta3b_eval(self._ctx, _p(w), num_models, self._nparams(w, num_models), _p(s), s.size,
                                        max_moves, _p(sc), _p(pc), _p(lc)))
        return sc, pc, lc

    def eval_islands(self, weights, seeds_per_island, max_moves: int):
        """weights (islands * models_per_island, 97); seeds_per_island (islands, games)."""
        s = np.ascontiguousarray(seeds_per_island, dtype=np.uint64)
        islands, games = s.shape
        w = _rows(weights)
        if w.shape[0] % islands:
            raise EvaluatorError("model count must be a multiple of the island count")
        mpi = w.shape[0] // islands
        n = w.shape[0] * games
        sc, pc, lc = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        self._check(self._lib.ta3b_eval_islands(self._ctx, _p(w), islands, mpi, w.shape[1], _p(s), games, max_moves,
                                                _p(sc), _p(pc), _p(lc)))
        return sc, pc, lc

    def eval_timed(self, weights, seeds_per_island, max_moves: int):
        """Island batch plus per-sim scheduling data: (score, pieces, evals, timing[n, 2] ns)."""
        s = np.ascontiguousarray(seeds_per_island, dtype=np.uint64)
        islands, games = s.shape
        w = _rows(weights)
        n = w.shape[0] * games
        sc, pc, ec = np.zeros(n, np.float32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        tm = np.zeros((n, 2), np.uint64)
        self._check(self._lib.ta3b_eval_timed(self._ctx, _p(w), islands, w.shape[0] // islands, w.shape[1], _p(s),
                                              games, max_moves, _p(sc), _p(pc), _p(ec), _p(tm)))
        return sc, pc, ec, tm

    def eval_trace(self, weights, num_models: int, seeds, max_moves: int, keys: bool = False):
        """Everything, plus per-move traces: dict of model-major arrays. keys=True adds
        "keys" (sims, max_moves, 2) uint64: each searched move's two largest final keys
        (decode with decode_key; see top2_margin)."""
        w, s = self._prep(weights, num_models, seeds)
        n = num_models * s.size
        out = {"score": np.zeros(n, np.float32), "pieces": np.zeros(n, np.uint32), "lines": np.zeros(n, np.uint32),
               "evals": np.zeros(n, np.uint32), "trace": np.zeros((n, max(max_moves, 1) * 3), np.uint8),
               "moves": np.zeros(n, np.uint32), "board": np.zeros((n, 10), np.uint32)}
        if keys:
            out["keys"] = np.zeros((n, max(max_moves, 1), 2), np.uint64)
        self._check(self._lib.ta3b_eval_trace(self._ctx, _p(w), num_models, self._nparams(w, num_models), _p(s), s.size,
                                              max_moves,
                                              _p(out["score"]), _p(out["pieces"]), _p(out["lines"]),
                                              _p(out["evals"]), _p(out["trace"]), _p(out["moves"]),
                                              _p(out["board"]), _p(out.get("keys"))))
        return out

    def eval_device(self, weights, seeds, max_moves: int, score, pieces=None, lines=None, evals=None,
                    num_islands: int = 1, stream=None):
        """Device-resident batch (torch CUDA tensors); enqueued, not synchronised.
        weights (islands * mpi, 97 or 4929) float32, seeds (islands, games) uint64 viewed as int64."""
        islands = num_islands
        games = seeds.numel() // islands
        nparams = weights.shape[-1] if weights.dim() == 2 and weights.shape[-1] in MODEL_SIZES else NUM_PARAMS
        models = weights.numel() // nparams
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        st = C.c_void_p(stream.cuda_stream) if stream is not None else None
        self._check(self._lib.ta3b_eval_device(self._ctx, ptr(weights), islands, models // islands, nparams,
                                               ptr(seeds), games, max_moves, ptr(score), ptr(pieces), ptr(lines),
                                               ptr(evals), st))

    def device_status(self) -> int:
        """Status word of the context's most recent launch (0 = no error); raises on a non-zero
        status. After eval_device, call it once the stream the batch ran on has finished."""
        st = C.c_uint32()
        self._check(self._lib.ta3b_device_status(self._ctx, C.byref(st)))
        return st.value

    def set_time_budget(self, seconds: float):
        """Per-launch time budget (0 = none): past it the call raises with an incomplete batch."""
        self._check(self._lib.ta3b_set_time_budget(self._ctx, float(seconds)))

    def select_variant(self, variant: int):
        self._check(self._lib.ta3b_select_variant(self._ctx, variant))

    def set_tail_handoff(self, on: bool):
        """Hand a full batch's tail to the paired kernel (default on); off keeps every game on one warp."""
        self._check(self._lib.ta3b_set_tail_handoff(self._ctx, int(bool(on))))

    def set_test_flags(self, flags: int):
        """Tests only: 1 = team partners leave at launch start (the leaders' waits run out)."""
        self._check(self._lib.ta3b_set_test_flags(self._ctx, flags))

    def handoff_games(self) -> int:
        """How many games the last launch handed to the paired kernel."""
        n = C.c_uint32()
        self._check(self._lib.ta3b_handoff_info(self._ctx, C.byref(n)))
        return n.value

    @staticmethod
    def variants():
        lib = library()
        out = []
        for v in range(lib.ta3b_num_variants()):
            w, b = C.c_uint32(), C.c_uint32()
            lib.ta3b_variant_info(v, C.byref(w), C.byref(b))
            out.append({"variant": v, "warps_per_block": w.value, "min_blocks_per_sm": b.value,
                        "warps_per_game": lib.ta3b_variant_warps_per_game(v)})
        return out

    def autotune(self, weights, seeds, max_moves: int, score, pieces=None, lines=None, evals=None,
                 num_islands: int = 1, stream=None, reps: int = 1):
        """Time every launch-shape variant on this device batch (CUDA events on
        `stream`) and keep the fastest. Returns {variant: ms}. A paired variant is
        timed only when one block per SM holds the batch (beyond that its games
        run in waves)."""
        import torch
        times = {}
        st = stream or torch.cuda.current_stream()
        sms = self.launch_info()["sms"]
        for info in self.variants():
            v = info["variant"]
            if info["warps_per_game"] > 1 and score.numel() > sms * info["warps_per_block"] // info["warps_per_game"]:
                continue
            self.select_variant(v)
            with torch.cuda.stream(st):
                self.eval_device(weights, seeds, max_moves, score, pieces, lines, evals, num_islands, st)  # warm
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                for _ in range(reps):
                    self.eval_device(weights, seeds, max_moves, score, pieces, lines, evals, num_islands, st)
                b.record(st)
            b.synchronize()
            times[v] = a.elapsed_time(b) / reps
        self.select_variant(min(times, key=times.get))
        return times

    def launch_info(self):
        g, w, s = C.c_uint32(), C.c_uint32(), C.c_uint32()
        k = C.c_uint32()
        self._check(self._lib.ta3b_launch_info(self._ctx, C.byref(g), C.byref(w), C.byref(s), C.byref(k)))
        return {"grid": g.value, "warps_per_block": w.value, "sms": s.value, "kernels": k.value}


def simulate(evaluator: ModelEvaluator, model_weights, num_models: int, games: int, seed: int,
             max_moves: int) -> np.ndarray:
    """ta3::gpu::simulate: games seeds drawn from xoshiro256**(seed), shared by every model."""
    return evaluator.eval(model_weights, num_models, simulate_seeds(seed, games), max_moves)


class GenerationGraph:
    """One CMA-ES generation's launch sequence captured as a CUDA graph:
    pinned host weights and seeds -> device, the evaluation kernel (work-queue
    reset + persistent launch), device results -> pinned host. Replaying it
    scores a new population of the same shape with one graph launch."""

    def __init__(self, evaluator: ModelEvaluator, models: int, islands: int, games: int, max_moves: int,
                 device: int = 0):
        import torch
        if models % islands:
            raise EvaluatorError("model count must be a multiple of the island count")
        self.torch = torch
        dev = torch.device("cuda", device)
        self.shape = (models, islands, games, max_moves)
        n = models * games
        self.h_w = torch.empty((models, NUM_PARAMS), dtype=torch.float32).pin_memory()
        self.h_s = torch.empty((islands, games), dtype=torch.int64).pin_memory()
        self.d_w = torch.empty((models, NUM_PARAMS), dtype=torch.float32, device=dev)
        self.d_s = torch.empty((islands, games), dtype=torch.int64, device=dev)
        self.d_out = [torch.empty(n, dtype=t, device=dev) for t in (torch.float32, torch.int32, torch.int32,
                                                                     torch.int32)]
        self.h_out = [torch.empty(n, dtype=t).pin_memory() for t in (torch.float32, torch.int32, torch.int32,
                                                                      torch.int32)]
        self.stream = torch.cuda.Stream(device=dev)
        self.graph = torch.cuda.CUDAGraph()
        self.h_w.zero_()
        self.h_s.zero_()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self.d_w.copy_(self.h_w, non_blocking=True)
            self.d_s.copy_(self.h_s, non_blocking=True)
            evaluator.eval_device(self.d_w, self.d_s, max_moves, *self.d_out, num_islands=islands,
                                  stream=self.stream)
            for h, d in zip(self.h_out, self.d_out):
                h.copy_(d, non_blocking=True)

    def run(self, weights, seeds_per_island):
        """Score one population: (score, pieces, lines, evaluated placements), model-major."""
        models, islands, games, _ = self.shape
        w = np.ascontiguousarray(weights, dtype=np.float32).reshape(models, NUM_PARAMS)
        s = np.ascontiguousarray(seeds_per_island, dtype=np.uint64).reshape(islands, games)
        self.h_w.numpy()[:] = w
        self.h_s.numpy()[:] = s.view(np.int64)
        # replay() launches on the current stream: make that the stream whose completion we wait for
        with self.torch.cuda.stream(self.stream):
            self.graph.replay()
        self.stream.synchronize()
        sc, pc, lc, ec = (h.numpy().copy() for h in self.h_out)
        return sc, pc.view(np.uint32), lc.view(np.uint32), ec.view(np.uint32)
