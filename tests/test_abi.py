"""The C-ABI library without a GPU: it loads, exports every function
include/ta3b.h declares, its host-only seed derivation equals the reference's,
the C++ drop-in header compiles and links against it, and without a device it
fails loudly (there is no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, ptr

HEADER = os.path.join(ROOT, "include", "ta3b.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ta3b_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from tetris_ai3_b200 import library
    return library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from tetris_ai3_b200.evaluator import EXPORTS
    assert sorted(EXPORTS) == declared_functions()


def test_simulate_seeds_match_reference(lib):
    g = load_golden("engine")["simulate_seeds"]
    for s, want in g.items():
        out = np.zeros(16, np.uint64)
        assert lib.ta3b_simulate_seeds(C.c_uint64(int(s)), 16, ptr(out)) == 0
        assert [str(int(v)) for v in out] == want
    from tetris_ai3_b200 import simulate_seeds, workload
    assert np.array_equal(simulate_seeds(42, 16), workload.xoshiro_seeds(42, 16))


def test_variants_enumerate(lib):
    from tetris_ai3_b200 import ModelEvaluator
    v = ModelEvaluator.variants()
    assert len(v) == lib.ta3b_num_variants() >= 2
    solo = [x for x in v if x["warps_per_game"] == 1]
    teams = [x for x in v if x["warps_per_game"] > 1]
    assert len(solo) + len(teams) == len(v) and teams
    assert {x["warps_per_block"] for x in solo} == {2, 4, 8, 10, 16, 20}
    assert {x["warps_per_game"] for x in teams} == {2, 4}
    assert all(x["warps_per_block"] % x["warps_per_game"] == 0 for x in teams)
    assert lib.ta3b_variant_warps_per_game(-1) == -1 and lib.ta3b_variant_warps_per_game(len(v)) == -1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_fails_loudly_without_a_device():
    from tetris_ai3_b200 import EvaluatorError, ModelEvaluator
    with pytest.raises(EvaluatorError):
        ModelEvaluator(device=0)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_dropin_header_compiles_and_links(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text(r'''
#include <ta3b.hpp>
#include <cstdio>
int main() {
    std::vector<float> w(97, 0.1f);
    std::vector<std::uint64_t> seeds{1, 2};
    try {
        ta3::gpu::ModelEvaluator ev;
        auto s = ta3::gpu::simulate(ev, w, 2, 7, 300);
        std::printf("ran %zu\n", s.size());
    } catch (std::runtime_error const& e) {
        std::printf("error %s\n", e.what());
    }
    return 0;
}
''')
    exe = tmp_path / "use"
    libdir = os.path.join(ROOT, "tetris_ai3_b200", "_lib")
    subprocess.run(["g++", "-std=c++20", "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir, "-lta3b",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120).stdout
    assert out.startswith("ran 7") if _has_gpu() else out.startswith("error ta3b:")


def _declared(header: str, prefix: str):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(rf"\b({prefix}[a-z0-9_]+)\s*\(", text)) - {"ta3t_score_fn"})


def test_host_library_exports_the_cma_and_trainer_headers(host):
    lib = host.host_library()
    names = _declared("ta3b_cma.h", "ta3c_") + _declared("ta3b_trainer.h", "ta3t_")
    assert len(names) >= 25
    assert [n for n in names if not hasattr(lib, n)] == []
    assert sorted(host.HOST_EXPORTS) == names


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_trainer_headers_compile_and_link(tmp_path):
    src = tmp_path / "use_trainer.cpp"
    src.write_text(r'''
#include <ta3b_cma.h>
#include <ta3b_trainer.h>
#include <cstdio>
#include <vector>
static int score(void*, const float* w, uint32_t n, uint32_t p, const uint64_t*, uint32_t g, uint32_t,
                 float* out, uint32_t*) {
    for (uint32_t m = 0; m < n; ++m) {
        double s = 0; for (uint32_t j = 0; j < p; ++j) s -= double(w[m * p + j]) * w[m * p + j];
        for (uint32_t k = 0; k < g; ++k) out[m * g + k] = float(s);
    }
    return 0;
}
int main() {
    ta3t_config c; ta3t_default_config(&c);
    c.islands = 2; c.population = 6; c.games = 2; c.gens_per_iteration = 2;
    ta3t_trainer* t = ta3t_create(&c, score, nullptr, nullptr);
    if (!t) { std::printf("error %s\n", ta3t_last_error(nullptr)); return 1; }
    ta3t_run(t, 2);
    ta3t_stats st; ta3t_get_stats(t, &st);
    std::printf("gens %llu\n", (unsigned long long)st.generation);
    ta3t_destroy(t);
    return 0;
}
''')
    exe = tmp_path / "use_trainer"
    libdir = os.path.join(ROOT, "tetris_ai3_b200", "_lib")
    subprocess.run(["g++", "-std=c++20", "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir, "-lta3b_host",
                    "-lta3b", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120).stdout
    assert out.startswith("gens 4"), out


def test_surrogate_header_is_exported():
    from tetris_ai3_b200 import library
    from tetris_ai3_b200.surrogate import SURROGATE_EXPORTS
    names = sorted(_declared("ta3b_surrogate.h", "ta3s_") + _declared("ta3b_surrogate.h", "ta3w_"))
    assert names == SURROGATE_EXPORTS
    lib = library()
    assert [n for n in names if not hasattr(lib, n)] == []


def test_noalloc_sim_bound_is_checked_before_any_device_call(lib):
    """The work queue's ticket is 64-bit and sim indices are 32-bit: a call may cover up to
    2^32 - 1 sims. The bound is checked on the host before anything touches a device."""
    err = C.c_char_p()
    # 65536 x 65536 x 1 = 2^32 sims: one too many
    rc = lib.ta3b_eval_device_noalloc(None, 65536, 65536, 97, None, 1, 10, None, None, None, None, None,
                                      C.byref(err))
    assert rc == -1 and b"too many sims" in err.value and b"2^32 - 1" in err.value
    # 65535 x 65537 x 1 = 2^32 - 1 sims: within the bound, so the next check (null pointers) answers
    rc = lib.ta3b_eval_device_noalloc(None, 65535, 65537, 97, None, 1, 10, None, None, None, None, None,
                                      C.byref(err))
    assert rc == -1 and b"null" in err.value
    assert lib.ta3b_noalloc_status(None, None, C.byref(err)) == -1 and b"null" in err.value


def test_status_query_rejects_a_null_context(lib):
    assert lib.ta3b_device_status(None, None) == -1


def test_context_settings_reject_a_null_context(lib):
    assert lib.ta3b_set_test_flags(None, 0) == -1
    assert lib.ta3b_set_tail_handoff(None, 1) == -1
    assert lib.ta3b_handoff_info(None, None) == -1
