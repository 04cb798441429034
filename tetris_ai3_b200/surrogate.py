"""Python binding of the GPU surrogate model (include/ta3b_surrogate.h, in
libta3b.so): an MLP in_dim -> hidden -> hidden -> 2 (97 -> 128 -> 128 -> 2 for
v11, 4929 -> 256 -> 256 -> 2 for the widened evaluator) trained on (parameter
vector -> mean score) pairs with hand-written tcgen05 forward / backward / Adam
kernels. `train(x, y)` / `predict(x)` make it usable as the island trainer's
surrogate."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .evaluator import EvaluatorError, library

_SIG = {
    "ta3s_num_params": (C.c_uint32, []),
    "ta3s_create": (C.c_void_p, [C.c_int, C.c_uint32]),
    "ta3s_destroy": (None, [C.c_void_p]),
    "ta3s_last_error": (C.c_char_p, [C.c_void_p]),
    "ta3s_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ta3s_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ta3s_set_data": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "ta3s_set_data_standardized": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "ta3s_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ta3s_train": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.c_void_p]),
    "ta3s_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    # any parameter-vector size (the widened evaluator's 4,929)
    "ta3w_num_params": (C.c_uint32, [C.c_uint32, C.c_uint32]),
    "ta3w_create": (C.c_void_p, [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32]),
    "ta3w_destroy": (None, [C.c_void_p]),
    "ta3w_last_error": (C.c_char_p, [C.c_void_p]),
    "ta3w_model_params": (C.c_uint32, [C.c_void_p]),
    "ta3w_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ta3w_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ta3w_set_data": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "ta3w_set_data_standardized": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "ta3w_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ta3w_train": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.c_void_p]),
    "ta3w_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "ta3w_gemm_test": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
}
SURROGATE_EXPORTS = sorted(_SIG)
V11_SHAPE = (97, 128)            # the fused single-kernel model (ta3s_*)


def _lib():
    lib = library()
    for name, (res, args) in _SIG.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Surrogate:
    """The GPU surrogate: in_dim -> hidden -> hidden -> 2. The v11 shape (97, 128)
    runs the fused kernel (ta3s_*); any other shape, e.g. the widened evaluator's
    (4929, 256), the layer-by-layer GEMM path (ta3w_*). Raises EvaluatorError
    without an sm_100 device."""

    def __init__(self, device: int = 0, seed: int = 0, epochs: int = 40, batch: int = 256, lr: float = 1e-3,
                 weight_decay: float = 0.0, in_dim: int = 97, hidden: int = 128):
        self.lib = _lib()
        self.in_dim, self.hidden = in_dim, hidden
        self.fused = (in_dim, hidden) == V11_SHAPE
        self._pre = "ta3s_" if self.fused else "ta3w_"
        if self.fused:
            self.h = self.lib.ta3s_create(device, seed)
        else:
            self.h = self.lib.ta3w_create(device, in_dim, hidden, seed)
        if not self.h:
            raise EvaluatorError(self._f("last_error")(None).decode())
        self.nparam = int(self.lib.ta3s_num_params() if self.fused else self.lib.ta3w_model_params(self.h))
        self.epochs, self.batch, self.lr, self.wd, self.seed = epochs, batch, lr, weight_decay, seed
        self.trainings = 0
        self.last_loss = float("nan")

    def _f(self, name):
        return getattr(self.lib, self._pre + name)

    def __del__(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def _ok(self, rc):
        if rc:
            raise EvaluatorError(self._f("last_error")(self.h).decode())

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        self._ok(self._f("get_params")(self.h, _p(out)))
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        self._ok(self._f("set_params")(self.h, _p(p)))

    def _set_data(self, x, y, standardized: bool):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        assert x.ndim == 2 and x.shape[1] == self.in_dim and len(y) == len(x)
        fn = self._f("set_data_standardized" if standardized else "set_data")
        self._ok(fn(self.h, _p(x), _p(y), len(y)))

    def gradients(self, x, y, standardized: bool = True):
        """Gradient of the mean loss over (x, y) and the summed loss, no update."""
        self._set_data(x, y, standardized)
        g = np.empty(self.nparam, np.float32)
        loss = C.c_float()
        self._ok(self._f("gradients")(self.h, _p(g), C.byref(loss)))
        return g, loss.value

    def train(self, x, y, epochs: int | None = None, batch: int | None = None, standardized: bool = False):
        self._set_data(x, y, standardized)
        loss = C.c_float()
        self._ok(self._f("train")(self.h, epochs or self.epochs, batch or self.batch, self.lr, self.wd,
                                  self.seed + self.trainings, C.byref(loss)))
        self.trainings += 1
        self.last_loss = loss.value
        return loss.value

    def predict(self, x, with_logvar: bool = False):
        x = np.ascontiguousarray(x, np.float32)
        n = len(x)
        mean = np.empty(n, np.float32)
        lv = np.empty(n, np.float32) if with_logvar else None
        self._ok(self._f("predict")(self.h, _p(x), n, _p(mean), _p(lv)))
        return (mean, lv) if with_logvar else mean


def gemm_test(a, b, a_mn: bool, b_mn: bool, m: int, n: int, k: int, splits: int = 1, device: int = 0):
    """The surrogate's tcgen05 GEMM kernel alone: a, b are BF16 bit patterns (uint16)
    in their global layouts; returns C [m][n] = sum_k A(m, k) B(n, k) (FP32)."""
    lib = _lib()
    a = np.ascontiguousarray(a, np.uint16)
    b = np.ascontiguousarray(b, np.uint16)
    c = np.empty((m, n), np.float32)
    if lib.ta3w_gemm_test(device, int(a_mn), int(b_mn), m, n, k, splits, _p(a), _p(b), _p(c)):
        raise EvaluatorError(lib.ta3w_last_error(None).decode())
    return c


def main(argv=None):
    """Time the GPU surrogate on a seeded synthetic (parameters -> score) set:
    python -m tetris_ai3_b200.surrogate [--rows 8000] [--epochs 40] [--batch 256]
                                        [--in-dim 97 --hidden 128 | --in-dim 4929 --hidden 256]"""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=8000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--predict", type=int, default=800)
    ap.add_argument("--in-dim", type=int, default=V11_SHAPE[0])
    ap.add_argument("--hidden", type=int, default=V11_SHAPE[1])
    args = ap.parse_args(argv)
    rng = np.random.default_rng(0)
    a = rng.normal(size=(8, args.in_dim)) / np.sqrt(args.in_dim)
    x = rng.normal(size=(args.rows, args.in_dim)).astype(np.float32)
    y = (-((x @ a.T) ** 2).sum(1)).astype(np.float32)
    s = Surrogate(batch=args.batch, epochs=args.epochs, in_dim=args.in_dim, hidden=args.hidden)
    s.train(x[:256], y[:256], epochs=1)                 # warm-up: first launches, buffers
    t0 = time.perf_counter()
    loss = s.train(x, y)
    t1 = time.perf_counter()
    s.predict(x[:args.predict])
    t2 = time.perf_counter()
    steps = args.epochs * ((args.rows + args.batch - 1) // args.batch)
    print(json.dumps({"in_dim": args.in_dim, "hidden": args.hidden, "params": s.nparam, "rows": args.rows,
                      "epochs": args.epochs, "batch": args.batch, "train_s": t1 - t0,
                      "ms_per_step": 1e3 * (t1 - t0) / steps, "predict_ms": 1e3 * (t2 - t1), "final_loss": loss}))


if __name__ == "__main__":
    main()
