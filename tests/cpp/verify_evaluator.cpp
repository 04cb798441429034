// The reference trainer's start-up self-check (ta3_trainer/src/trainer2.cpp:57-89), written
// against the C++ drop-in header: 2 models with weights drawn uniformly from the v11 bounds
// [-2, 2] by xoshiro256**(0xC0FFEE) (one draw per weight, rng() >> 11 scaled by 2^-53), seeds
// {101, 202, 303}, 100 moves. ModelEvaluator::eval runs on the GPU (libta3b.so);
// ModelEvaluator::eval_host runs the reference's own CPU search (integration/ta3b_eval_host.cpp,
// linked into this program as a trainer would link it).
//
// Prints one line per (model, game) with both scores' bit patterns, then "parity ok" or
// "parity FAIL". With "--host-only" it skips the device (a CPU-only check of the host side).
#include <ta3b.hpp>

#include <array>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

namespace {

std::uint32_t bits(float f) {
    std::uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

} // namespace

int main(int argc, char** argv) {
    bool const host_only = argc > 1 && std::strcmp(argv[1], "--host-only") == 0;
    constexpr std::uint32_t MODELS = 2, GAMES = 3, MOVES = 100, P = TA3B_NUM_PARAMS;
    constexpr double LO = -2.0, HI = 2.0;   // model_v11.hpp:41 BOUNDS

    // xoshiro256**(0xC0FFEE) draws: the same generator ta3::gpu::simulate seeds games with
    std::vector<std::uint64_t> draws(MODELS * P);
    if (ta3b_simulate_seeds(0xC0FFEEull, MODELS * P, draws.data()) != TA3B_OK) return 2;
    std::vector<ta3::gpu::weights_t> w(MODELS * P);
    for (std::size_t i = 0; i < w.size(); ++i)
        w[i] = static_cast<ta3::gpu::weights_t>(LO + (HI - LO) * (static_cast<double>(draws[i] >> 11) * 0x1.0p-53));
    std::array<std::uint64_t, GAMES> const seeds{101, 202, 303};

    std::vector<std::vector<float>> host(MODELS);
    for (std::uint32_t m = 0; m < MODELS; ++m)
        host[m] = ta3::gpu::ModelEvaluator::eval_host(std::span{w}.subspan(m * P, P), seeds, MOVES);
    if (host_only) {
        for (std::uint32_t m = 0; m < MODELS; ++m)
            for (std::uint32_t g = 0; g < GAMES; ++g) std::printf("host %u %u %08x\n", m, g, bits(host[m][g]));
        return 0;
    }

    std::vector<float> dev;
    try {
        ta3::gpu::ModelEvaluator evaluator;
        dev = evaluator.eval(w, MODELS, seeds, MOVES);
    } catch (std::exception const& e) {
        std::printf("error %s\n", e.what());
        return 3;
    }
    bool ok = dev.size() == MODELS * GAMES;
    for (std::uint32_t m = 0; ok && m < MODELS; ++m)
        for (std::uint32_t g = 0; g < GAMES; ++g) {
            float const d = dev[m * GAMES + g], h = host[m][g];
            std::printf("model %u game %u device %08x host %08x\n", m, g, bits(d), bits(h));
            ok = ok && bits(d) == bits(h);
        }
    // trainer2.cpp:79-81: two distinct models must not score identically
    bool const distinct = std::memcmp(dev.data(), dev.data() + GAMES, GAMES * sizeof(float)) != 0;
    std::printf("%s%s\n", ok ? "parity ok" : "parity FAIL", distinct ? "" : " (models scored identically)");
    return ok && distinct ? 0 : 1;
}
