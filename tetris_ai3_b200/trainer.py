"""Python binding of the C++ host side: the CMA-ES optimisers
(include/ta3b_cma.h) and the island trainer (include/ta3b_trainer.h), both in
tetris_ai3_b200/_lib/libta3b_host.so.

The trainer restates ta3::trn::Trainer2 (ta3_trainer/src/trainer2.cpp): it
scores every island's generation in one call of the GPU evaluator (or of a
score function given here, e.g. for CPU tests) and can pre-screen candidates
with a surrogate model.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Callable, Optional

import numpy as np

from .evaluator import NUM_PARAMS

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libta3b_host.so")
_lib = None

SEP, DD = 1, 2

SCORE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64),
                       C.c_uint32, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_uint32))
TRAIN_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32, C.c_uint32)
PREDICT_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.POINTER(C.c_float))


class TrainerConfig(C.Structure):
    _fields_ = [("islands", C.c_uint32), ("population", C.c_uint32), ("gens_per_iteration", C.c_uint32),
                ("iterations_per_cycle", C.c_uint32), ("games", C.c_uint32), ("max_moves", C.c_uint32),
                ("algo", C.c_uint32), ("num_params", C.c_uint32), ("training_seed", C.c_uint64),
                ("sigma0", C.c_double), ("lower", C.c_double), ("upper", C.c_double), ("device", C.c_int),
                ("surrogate_start_gen", C.c_uint32), ("surrogate_sample", C.c_uint32),
                ("surrogate_top", C.c_uint32), ("surrogate_random", C.c_uint32),
                ("surrogate_retrain", C.c_uint32), ("surrogate_min_rho", C.c_double),
                ("surrogate_epochs", C.c_uint32), ("surrogate_batch", C.c_uint32), ("surrogate_lr", C.c_double),
                ("surrogate_window", C.c_uint32), ("num_devices", C.c_uint32)]


class TrainerStats(C.Structure):
    _fields_ = [("generation", C.c_uint64), ("iteration", C.c_uint64), ("evaluations", C.c_uint64),
                ("sims", C.c_uint64), ("pieces", C.c_uint64), ("game_seed", C.c_uint64),
                ("best_fitness", C.c_double), ("eval_seconds", C.c_double), ("host_seconds", C.c_double),
                ("surrogate_seconds", C.c_double), ("last_rho", C.c_double), ("surrogate_active", C.c_uint32),
                ("surrogate_trainings", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SurrogateStruct(C.Structure):
    _fields_ = [("user", C.c_void_p), ("train", TRAIN_FN), ("predict", PREDICT_FN)]


def host_library() -> C.CDLL:
    """libta3b_host.so (built by tetris_ai3_b200.build.build_host)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB):
        raise RuntimeError(f"{_LIB} is missing: run python -m tetris_ai3_b200.build")
    lib = C.CDLL(_LIB)
    vp, u32, u64, dbl, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double, C.c_int
    sig = {
        "ta3c_create": (vp, [i32, u32, vp, vp, vp, dbl, u32, i32]),
        "ta3c_destroy": (None, [vp]),
        "ta3c_new_evolve": (i32, [vp]),
        "ta3c_ask": (i32, [vp, u32, vp]),
        "ta3c_last_dx": (dbl, [vp]),
        "ta3c_tell": (i32, [vp, u32, vp, vp]),
        "ta3c_mean": (i32, [vp, vp]),
        "ta3c_sigma": (dbl, [vp]),
        "ta3c_axis_std": (i32, [vp, vp]),
        "ta3c_whiten": (i32, [vp, u32, vp, vp]),
        "ta3c_dim": (u32, [vp]),
        "ta3c_save": (u64, [vp, vp, u64]),
        "ta3c_load": (vp, [vp, u64]),
        "ta3c_last_error": (C.c_char_p, []),
        "ta3c_sym_eig": (i32, [u32, vp, vp, vp]),
        "ta3c_run_test_problem": (i32, [i32, i32, u32, u32, u32, dbl, u32, dbl, dbl, vp, vp]),
        "ta3t_default_config": (None, [C.POINTER(TrainerConfig)]),
        "ta3t_create": (vp, [C.POINTER(TrainerConfig), SCORE_FN, vp, C.POINTER(SurrogateStruct)]),
        "ta3t_create_from_state": (vp, [C.POINTER(TrainerConfig), C.c_char_p, SCORE_FN, vp,
                                        C.POINTER(SurrogateStruct)]),
        "ta3t_create_groups": (vp, [C.POINTER(TrainerConfig), u32, vp, vp, C.POINTER(SurrogateStruct)]),
        "ta3t_destroy": (None, [vp]),
        "ta3t_last_error": (C.c_char_p, [vp]),
        "ta3t_next_game_seed": (i32, [vp]),
        "ta3t_run_generation": (i32, [vp]),
        "ta3t_run_iteration": (i32, [vp]),
        "ta3t_run": (i32, [vp, u32]),
        "ta3t_get_stats": (i32, [vp, C.POINTER(TrainerStats)]),
        "ta3t_champion": (i32, [vp, u32, vp, vp]),
        "ta3t_island_mean": (i32, [vp, u32, vp]),
        "ta3t_island_whiten": (i32, [vp, u32, vp, u32, vp]),
        "ta3t_save_state": (i32, [vp, C.c_char_p]),
        "ta3t_write_champ": (i32, [C.c_char_p, vp, u64]),
        "ta3t_read_champ": (u64, [C.c_char_p, vp, u64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


HOST_EXPORTS = ["ta3c_create", "ta3c_destroy", "ta3c_new_evolve", "ta3c_ask", "ta3c_last_dx", "ta3c_tell",
                "ta3c_mean", "ta3c_sigma", "ta3c_axis_std", "ta3c_whiten", "ta3c_dim", "ta3c_save", "ta3c_load",
                "ta3c_last_error", "ta3c_sym_eig", "ta3c_run_test_problem", "ta3t_default_config", "ta3t_create",
                "ta3t_create_from_state", "ta3t_create_groups", "ta3t_destroy", "ta3t_last_error", "ta3t_next_game_seed",
                "ta3t_run_generation", "ta3t_run_iteration", "ta3t_run", "ta3t_get_stats", "ta3t_champion",
                "ta3t_island_mean", "ta3t_island_whiten", "ta3t_save_state", "ta3t_write_champ", "ta3t_read_champ"]


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Cma:
    """sep-CMA-ES (kind=SEP) or dd-CMA-ES (kind=DD) as an ask/tell optimiser."""

    def __init__(self, kind: int, x0, lb, ub, sigma0: float, seed: int, active: bool = True, _handle=None):
        self.lib = host_library()
        if _handle is not None:
            self.h = _handle
        else:
            x0 = np.ascontiguousarray(x0, np.float64)
            lb = np.ascontiguousarray(lb, np.float64)
            ub = np.ascontiguousarray(ub, np.float64)
            self.h = self.lib.ta3c_create(kind, len(x0), _p(x0), _p(lb), _p(ub), sigma0, seed, int(active))
            if not self.h:
                raise ValueError(self.lib.ta3c_last_error().decode())
        self.dim = int(self.lib.ta3c_dim(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ta3c_destroy(self.h)
            self.h = None

    def _ok(self, rc):
        if rc:
            raise ValueError(self.lib.ta3c_last_error().decode())

    def new_evolve(self):
        self._ok(self.lib.ta3c_new_evolve(self.h))

    def ask(self, lam: int) -> np.ndarray:
        out = np.empty((lam, self.dim), np.float64)
        self._ok(self.lib.ta3c_ask(self.h, lam, _p(out)))
        return out

    def tell(self, fitness, idx=None):
        f = np.ascontiguousarray(fitness, np.float64)
        ix = None if idx is None else np.ascontiguousarray(idx, np.int32)
        self._ok(self.lib.ta3c_tell(self.h, len(f), None if ix is None else _p(ix), _p(f)))

    @property
    def mean(self) -> np.ndarray:
        out = np.empty(self.dim)
        self._ok(self.lib.ta3c_mean(self.h, _p(out)))
        return out

    @property
    def sigma(self) -> float:
        return float(self.lib.ta3c_sigma(self.h))

    def axis_std(self) -> np.ndarray:
        out = np.empty(self.dim)
        self._ok(self.lib.ta3c_axis_std(self.h, _p(out)))
        return out

    def whiten(self, x) -> np.ndarray:
        """Points (k, dim) in the coordinates where the current search distribution is N(0, I)."""
        x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
        z = np.empty_like(x)
        self._ok(self.lib.ta3c_whiten(self.h, x.shape[0], _p(x), _p(z)))
        return z

    @property
    def last_dx(self) -> float:
        return float(self.lib.ta3c_last_dx(self.h))

    def save(self) -> bytes:
        n = self.lib.ta3c_save(self.h, None, 0)
        buf = C.create_string_buffer(n)
        self.lib.ta3c_save(self.h, buf, n)
        return buf.raw

    @classmethod
    def load(cls, blob: bytes) -> "Cma":
        lib = host_library()
        h = lib.ta3c_load(blob, len(blob))
        if not h:
            raise ValueError(lib.ta3c_last_error().decode())
        return cls(0, None, None, None, 0.0, 0, _handle=h)


def run_test_problem(kind: int, problem: int, gens: int, dim: int = 10, pop: int = 12, sigma0: float = 0.5,
                     seed: int = 0xdd5, ftol: float = 1e-14, xtol: float = 1e-14):
    """The reference's optimiser test problems (0 sphere, 1 separable ellipsoid,
    2 rotated ellipsoid) run natively; returns (champion_f, champion_x)."""
    lib = host_library()
    f = C.c_double()
    x = np.empty(dim)
    rc = lib.ta3c_run_test_problem(kind, problem, dim, pop, gens, sigma0, seed, ftol, xtol, C.byref(f), _p(x))
    if rc:
        raise ValueError(lib.ta3c_last_error().decode())
    return f.value, x


def sym_eig(a: np.ndarray):
    lib = host_library()
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    w = np.empty(n)
    v = np.empty((n, n))
    rc = lib.ta3c_sym_eig(n, _p(a), _p(w), _p(v))
    return w, v, rc == 0


def default_config(**overrides) -> TrainerConfig:
    cfg = TrainerConfig()
    host_library().ta3t_default_config(C.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


ScoreCallable = Callable[[np.ndarray, np.ndarray, int], "np.ndarray | tuple[np.ndarray, np.ndarray]"]


class Trainer:
    """The island CMA-ES trainer. `score(weights (n, P) float32, seeds (G,)
    uint64, max_moves) -> scores (n, G)` (optionally also pieces) replaces the
    GPU evaluator when given; a list of such functions splits the islands into
    groups (island i to score[i % len(score)], the groups on concurrent host
    threads); `surrogate` is any object with `train(x, y)` and
    `predict(x) -> mean score`."""

    def __init__(self, config: Optional[TrainerConfig] = None, score=None,
                 surrogate=None, state_path: Optional[str] = None, **overrides):
        self.lib = host_library()
        self.cfg = config if config is not None else default_config()
        for k, v in overrides.items():
            setattr(self.cfg, k, v)
        self._keep = []
        self.calls = []          # (num_models, num_games, max_moves) of every score call
        groups = list(score) if isinstance(score, (list, tuple)) else None
        fn = SCORE_FN()
        if score is not None and groups is None:
            fn = SCORE_FN(self._wrap_score(score))
        self._keep.append(fn)
        sp = None
        if surrogate is not None:
            s = SurrogateStruct(None, TRAIN_FN(self._wrap_train(surrogate)), PREDICT_FN(self._wrap_predict(surrogate)))
            self._keep.append(s)
            sp = C.byref(s)
        if groups is not None:
            if state_path is not None:
                raise ValueError("island groups start from fresh populations")
            fns = (SCORE_FN * len(groups))(*[SCORE_FN(self._wrap_score(g)) for g in groups])
            self._keep.append(fns)
            self.h = self.lib.ta3t_create_groups(C.byref(self.cfg), len(groups), C.cast(fns, C.c_void_p), None, sp)
        elif state_path is None:
            self.h = self.lib.ta3t_create(C.byref(self.cfg), fn, None, sp)
        else:
            self.h = self.lib.ta3t_create_from_state(C.byref(self.cfg), state_path.encode(), fn, None, sp)
        if not self.h:
            raise RuntimeError(self.lib.ta3t_last_error(None).decode())

    def _wrap_score(self, score):
        def cb(_user, w, n, p, seeds, g, max_moves, out, pieces):
            try:
                W = np.ctypeslib.as_array(w, (n, p)).copy()
                S = np.ctypeslib.as_array(seeds, (g,)).copy()
                self.calls.append((n, g, max_moves))
                res = score(W, S, max_moves)
                sc, pc = (res if isinstance(res, tuple) else (res, None))
                np.ctypeslib.as_array(out, (n * g,))[:] = np.asarray(sc, np.float32).reshape(-1)
                if pieces and pc is not None:
                    np.ctypeslib.as_array(pieces, (n * g,))[:] = np.asarray(pc, np.uint32).reshape(-1)
                elif pieces:
                    np.ctypeslib.as_array(pieces, (n * g,))[:] = 0
                return 0
            except Exception as e:  # reported as a failed score call
                self.error = e
                return 1
        return cb

    def _wrap_train(self, sur):
        def cb(_user, x, y, n, d):
            try:
                sur.train(np.ctypeslib.as_array(x, (n, d)).copy(), np.ctypeslib.as_array(y, (n,)).copy())
                return 0
            except Exception as e:
                self.error = e
                return 1
        return cb

    def _wrap_predict(self, sur):
        def cb(_user, x, n, d, out):
            try:
                np.ctypeslib.as_array(out, (n,))[:] = np.asarray(
                    sur.predict(np.ctypeslib.as_array(x, (n, d)).copy()), np.float32)
                return 0
            except Exception as e:
                self.error = e
                return 1
        return cb

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ta3t_destroy(self.h)
            self.h = None

    def _ok(self, rc):
        if rc:
            raise RuntimeError(self.lib.ta3t_last_error(self.h).decode())

    def next_game_seed(self):
        self._ok(self.lib.ta3t_next_game_seed(self.h))

    def run_generation(self):
        self._ok(self.lib.ta3t_run_generation(self.h))

    def run_iteration(self):
        self._ok(self.lib.ta3t_run_iteration(self.h))

    def run(self, iterations: int):
        self._ok(self.lib.ta3t_run(self.h, iterations))

    def stats(self) -> dict:
        st = TrainerStats()
        self._ok(self.lib.ta3t_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def champion(self, island: int):
        x = np.empty(self.cfg.num_params)
        f = C.c_double()
        self._ok(self.lib.ta3t_champion(self.h, island, _p(x), C.byref(f)))
        return x, f.value

    def island_mean(self, island: int) -> np.ndarray:
        x = np.empty(self.cfg.num_params)
        self._ok(self.lib.ta3t_island_mean(self.h, island, _p(x)))
        return x

    def island_whiten(self, island: int, x) -> np.ndarray:
        """Parameter vectors (n, P) in the island's own search coordinates (its sampling
        distribution is N(0, I) there)."""
        x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
        z = np.empty_like(x)
        self._ok(self.lib.ta3t_island_whiten(self.h, island, _p(x), x.shape[0], _p(z)))
        return z

    def save_state(self, path: str):
        self._ok(self.lib.ta3t_save_state(self.h, path.encode()))


def write_champ(path: str, x) -> None:
    x = np.ascontiguousarray(x, np.float64)
    if host_library().ta3t_write_champ(path.encode(), _p(x), len(x)):
        raise OSError(f"cannot write {path}")


def read_champ(path: str) -> np.ndarray:
    lib = host_library()
    n = lib.ta3t_read_champ(path.encode(), None, 0)
    if n == 0:
        raise OSError(f"cannot read {path}")
    x = np.empty(n)
    lib.ta3t_read_champ(path.encode(), _p(x), n)
    return x


__all__ = ["Cma", "SEP", "DD", "Trainer", "TrainerConfig", "default_config", "run_test_problem", "sym_eig",
           "write_champ", "read_champ", "host_library", "NUM_PARAMS"]
