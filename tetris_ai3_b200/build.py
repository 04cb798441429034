"""In-tree build of the CUDA library (sm_100a) and of the oracle's C code.

    python -m tetris_ai3_b200.build          # builds tetris_ai3_b200/_lib/libta3b.so

The library is a plain C-ABI shared object (include/ta3b.h) compiled by nvcc
for sm_100a only; it travels with the repository snapshot, so nothing is
JIT-compiled at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libta3b.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: every floating-point operation on the evaluation path must round
# exactly like the reference CPU path (separate multiply and add); the source
# also spells the roundings out with __fmul_rn / __fadd_rn.
NVCC_FLAGS = ["-O3", "-std=c++20", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"]
SOURCES = ["ta3b_eval.cu", "ta3s_surrogate.cu", "ta3s_wide.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build_lib(verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", LIB + ".tmp", *srcs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return res.stderr


CORETEST_LIB = os.path.join(LIBDIR, "libta3b_coretest.so")


def build_coretest() -> str:
    """Host build of csrc/eval_core.h for the CPU tests (never loaded by the product)."""
    os.makedirs(LIBDIR, exist_ok=True)
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++20", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-I", CSRC,
           "-o", CORETEST_LIB, os.path.join(CSRC, "core_selftest.cpp")]
    subprocess.run(cmd, check=True)
    return CORETEST_LIB


HOSTDIR = os.path.join(PKG, "host")
HOST_LIB = os.path.join(LIBDIR, "libta3b_host.so")
HOST_SOURCES = ["cmaes.cpp", "cma_abi.cpp", "trainer.cpp"]


def build_host() -> str:
    """The C++ host side (CMA-ES, island trainer) as libta3b_host.so, linked
    against libta3b.so (the GPU evaluator) with an $ORIGIN rpath."""
    os.makedirs(LIBDIR, exist_ok=True)
    # the system g++ (TA3B_CXX overrides): a CXX wrapper that swaps GCC's
    # internal paths produced a library whose iostream calls crashed in-process
    cxx = os.environ.get("TA3B_CXX") or shutil.which("g++") or "g++"
    srcs = [os.path.join(HOSTDIR, s) for s in HOST_SOURCES]
    cmd = [cxx, "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           "-o", HOST_LIB + ".tmp", *srcs, "-L", LIBDIR, "-lta3b", "-Wl,-rpath,$ORIGIN", "-pthread"]
    subprocess.run(cmd, check=True)
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    return HOST_LIB


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


def build_reference_cpu(ref: str | None = None) -> bool:
    """Compile the reference's own CPU path into oracle/_ref from the checkout
    at `ref` (default: the TA3_REFERENCE environment variable). Without a
    checkout nothing is built and the prebuilt library, if any, is used."""
    ref = ref or os.environ.get("TA3_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "ta3_sim")):
        return False
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={ref}", "ref"], check=True)
    return True


if __name__ == "__main__":
    log = build_lib(verbose=True)
    build_host()
    build_coretest()
    build_oracle()
    build_reference_cpu()
    print("built", LIB)
