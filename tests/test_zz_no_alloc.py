"""The allocation-free entry point (ta3b_eval_device_noalloc) against the
context-based device entry point, through the C ABI.

It exists for callers that must not call cudaMalloc where they evaluate -- a
host framework whose pooling allocator owns all device memory, or a scheduler
thread that cannot take cudaMalloc's implicit device synchronisation. Its only
scratch is a static device array shared by every call, so this test runs it
twice in a row (the second call must not see the first call's work-queue
state) and compares both with ta3b_eval_device bit for bit. This file is
collected last so a failure here cannot hide the other tests' results."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev_outputs(torch, n, dev):
    return [torch.zeros(n, dtype=t, device=dev) for t in (torch.float32, torch.int32, torch.int32, torch.int32)]


def test_noalloc_matches_context_path_twice():
    import torch
    from tetris_ai3_b200 import ModelEvaluator, library, workload
    lib = library()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    b = workload.generation_batch(islands=2, pop=6, games=8, max_moves=160, seed=21)
    w = torch.from_numpy(b.weights).to(dev)
    s = torch.from_numpy(b.seeds.view(np.int64)).to(dev)
    n = b.sims
    ptr = lambda t: C.c_void_p(t.data_ptr())

    ev = ModelEvaluator(device=0)
    ref = _dev_outputs(torch, n, dev)
    stream = torch.cuda.current_stream(dev)
    ev.eval_device(w, s, b.max_moves, *ref, num_islands=b.islands, stream=stream)
    torch.cuda.synchronize()
    assert int(ref[1].sum()) > 0

    for call in range(2):
        out = _dev_outputs(torch, n, dev)
        err = C.c_char_p()
        rc = lib.ta3b_eval_device_noalloc(ptr(w), b.islands, b.models // b.islands, 97, ptr(s), b.games, b.max_moves,
                                          ptr(out[0]), ptr(out[1]), ptr(out[2]), ptr(out[3]),
                                          C.c_void_p(stream.cuda_stream), C.byref(err))
        assert rc == 0, err.value
        status = C.c_uint32(0xFFFFFFFF)
        assert lib.ta3b_noalloc_status(C.c_void_p(stream.cuda_stream), C.byref(status), C.byref(err)) == 0, err.value
        assert status.value == 0
        torch.cuda.synchronize()
        for a, r in zip(out, ref):
            assert torch.equal(a.view(torch.int32), r.view(torch.int32)), f"call {call}"
    assert ev.device_status() == 0
    ev.close()


def test_noalloc_rejects_oversized_and_bad_arguments():
    import torch
    from tetris_ai3_b200 import library
    lib = library()
    torch.cuda.set_device(0)
    w = torch.zeros(97, dtype=torch.float32, device="cuda")
    s = torch.zeros(1, dtype=torch.int64, device="cuda")
    o = torch.zeros(1, dtype=torch.float32, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    err = C.c_char_p()
    # 2^32 sims: one more than a call may cover (sim indices are 32-bit)
    rc = lib.ta3b_eval_device_noalloc(ptr(w), 65536, 65536, 97, ptr(s), 1, 10, ptr(o), None, None, None, None,
                                      C.byref(err))
    assert rc != 0 and b"too many sims" in err.value
    rc = lib.ta3b_eval_device_noalloc(ptr(w), 1, 1, 96, ptr(s), 1, 10, ptr(o), None, None, None, None, C.byref(err))
    assert rc != 0 and b"num_params" in err.value
    rc = lib.ta3b_eval_device_noalloc(None, 1, 1, 97, ptr(s), 1, 10, ptr(o), None, None, None, None, C.byref(err))
    assert rc != 0 and b"null" in err.value
