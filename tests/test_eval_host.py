"""ModelEvaluator::eval_host through the C++ drop-in (include/ta3b.hpp).

eval_host is the reference trainer's CPU parity path (ta3_gpu/incl/ta3/gpu/model_eval.hpp:62-67,
ta3_gpu/src/common/model_eval_host.cpp:26-53), called by its start-up self-check
(ta3_trainer/src/trainer2.cpp:57-89). Here it forwards to ta3b_eval_host, defined in
integration/ta3b_eval_host.cpp: caller-side code built against the reference's headers, never
part of libta3b.so. oracle/Makefile builds it as oracle/_ref/libta3b_eval_host.so.

CPU: libta3b.so and the package do not contain it; the caller-side build reproduces the
reference's own self-check and parity games (golden vectors); the self-check program compiles.
GPU: the self-check program runs verifyEvaluator's exact case, device == eval_host bit for bit.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, ptr, weights_from_hex

HOST_REF_SO = os.path.join(ROOT, "oracle", "_ref", "libta3b_eval_host.so")
LIBDIR = os.path.join(ROOT, "tetris_ai3_b200", "_lib")
PROGRAM = os.path.join(ROOT, "tests", "cpp", "verify_evaluator.cpp")

needs_host_ref = pytest.mark.skipif(not os.path.exists(HOST_REF_SO),
                                    reason="oracle/_ref/libta3b_eval_host.so not built (needs the reference checkout)")


def _exported(so: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.skipif(shutil.which("nm") is None, reason="needs nm")
def test_product_libraries_do_not_contain_eval_host():
    from tetris_ai3_b200 import library
    library()                                   # builds libta3b.so if absent
    for so in glob.glob(os.path.join(LIBDIR, "*.so")):
        names = _exported(so)
        assert "ta3b_eval_host" not in names, so
    assert "ta3b_eval" in _exported(os.path.join(LIBDIR, "libta3b.so"))


def test_package_never_names_eval_host():
    for path in glob.glob(os.path.join(ROOT, "tetris_ai3_b200", "**", "*.*"), recursive=True):
        if path.endswith((".py", ".cu", ".h", ".cpp", ".hpp")):
            assert "ta3b_eval_host" not in open(path).read(), path


def _case(name_prefix: str):
    return next(c for c in load_golden("games")["cases"] if c["name"].startswith(name_prefix))


def _host_ref():
    lib = C.CDLL(HOST_REF_SO)
    lib.ta3b_eval_host.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
    return lib


@needs_host_ref
@pytest.mark.parametrize("case", ["trainer self-check", "parity_test model seed 11"])
def test_caller_side_eval_host_reproduces_reference_games(case):
    c = _case(case)
    w = weights_from_hex(c["weights"]).reshape(-1, 97)
    seeds = np.array([int(s) for s in c["seeds"]], np.uint64)
    lib = _host_ref()
    for m in range(w.shape[0]):
        sc = np.zeros(seeds.size, np.float32)
        pc = np.zeros(seeds.size, np.uint32)
        lc = np.zeros(seeds.size, np.uint32)
        wm = np.ascontiguousarray(w[m])
        assert lib.ta3b_eval_host(ptr(wm), 97, ptr(seeds), seeds.size, c["max_moves"], ptr(sc), ptr(pc), ptr(lc)) == 0
        want = c["results"][m]
        assert [f"{int(x):08x}" for x in sc.view(np.uint32)] == [g["score"] for g in want]
        assert pc.tolist() == [g["pieces"] for g in want]
        assert lc.tolist() == [g["lines"] for g in want]


@needs_host_ref
def test_caller_side_eval_host_rejects_bad_arguments():
    lib = _host_ref()
    w = np.zeros(97, np.float32)
    seeds = np.array([1], np.uint64)
    sc = np.zeros(1, np.float32)
    assert lib.ta3b_eval_host(ptr(w), 96, ptr(seeds), 1, 10, ptr(sc), None, None) == -1
    assert lib.ta3b_eval_host(None, 97, ptr(seeds), 1, 10, ptr(sc), None, None) == -1
    assert lib.ta3b_eval_host(ptr(w), 97, ptr(seeds), 0, 10, None, None, None) == 0


def _compile(tmp_path) -> str:
    exe = str(tmp_path / "verify_evaluator")
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), PROGRAM, HOST_REF_SO,
                    "-L", LIBDIR, "-lta3b", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


@needs_host_ref
@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_self_check_program_host_side_matches_reference(tmp_path):
    """The program's weights are the trainer's (xoshiro256**(0xC0FFEE) in [-2, 2]); its host side
    equals the reference's own eval_host on them (golden self-check case)."""
    from tetris_ai3_b200 import library
    library()
    out = subprocess.run([_compile(tmp_path), "--host-only"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    got = [line.split()[-1] for line in out.stdout.splitlines() if line.startswith("host ")]
    want = [g["score"] for row in _case("trainer self-check")["results"] for g in row]
    assert got == want


@pytest.mark.gpu
@needs_host_ref
@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_self_check_program_device_equals_eval_host(tmp_path):
    """verifyEvaluator's case through ta3b.hpp: ModelEvaluator::eval (B200) == eval_host, bit for bit."""
    out = subprocess.run([_compile(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and "parity ok" in out.stdout, out.stdout + out.stderr
    lines = [line for line in out.stdout.splitlines() if line.startswith("model ")]
    assert len(lines) == 6
    want = [g["score"] for row in _case("trainer self-check")["results"] for g in row]
    assert [line.split()[5] for line in lines] == want
