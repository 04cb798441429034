// ta3b.hpp -- header-only C++ drop-in for ta3::gpu::ModelEvaluator over the C ABI (ta3b.h).
//
// Same class name, member signatures, argument meaning and error behaviour
// (std::runtime_error) as the reference's ta3_gpu/incl/ta3/gpu/model_eval.hpp:27-114, so
// ta3_trainer's TetrisProblem2::evalBatch (ta3_trainer/src/tetris_problem2.cpp:44-72) and
// Trainer2::verifyEvaluator (ta3_trainer/src/trainer2.cpp:57-89) compile against it unchanged.
//
// eval (the GPU path) calls libta3b.so. eval_host (the CPU parity path) forwards to
// ta3b_eval_host (ta3b_host_ref.h), which libta3b.so does NOT contain: the caller compiles
// integration/ta3b_eval_host.cpp into its own binary against the reference's headers, as the
// reference compiles ta3_gpu/src/common/model_eval_host.cpp. A caller that never calls
// eval_host needs neither.
#pragma once
#include "ta3b.h"
#include "ta3b_host_ref.h"

#include <cstdint>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

namespace ta3::gpu {

using weights_t = float;

class ModelEvaluator {
public:
    explicit ModelEvaluator(int device = 0) {
        ta3b_config const cfg{device, 0, 0};
        _ctx.reset(ta3b_create(&cfg));
        if (!_ctx) throw std::runtime_error(std::string("ta3b: ") + ta3b_last_error(nullptr));
    }

    // model_eval.hpp:46-51: per-(model, game) fitness, model-major
    [[nodiscard]] std::vector<float> eval(std::span<weights_t const> weights, std::uint32_t num_models,
                                          std::span<std::uint64_t const> seeds, std::uint32_t max_moves) {
        std::vector<float> out(static_cast<std::size_t>(num_models) * seeds.size());
        if (weights.size() != static_cast<std::size_t>(num_models) * TA3B_NUM_PARAMS)
            throw std::runtime_error("ta3b: eval: weights.size() must equal num_models * NUM_PARAMS");
        check(ta3b_eval(_ctx.get(), weights.data(), num_models, TA3B_NUM_PARAMS, seeds.data(),
                        static_cast<std::uint32_t>(seeds.size()), max_moves, out.data(), nullptr, nullptr));
        return out;
    }

    // model_eval.hpp:54-59: single-model convenience
    [[nodiscard]] std::vector<float> eval(std::span<weights_t const> weights, std::span<std::uint64_t const> seeds,
                                          std::uint32_t max_moves) {
        return eval(weights, 1u, seeds, max_moves);
    }

    // model_eval.hpp:62-67: the same games on the CPU, the parity reference for eval; reads the
    // first NUM_PARAMS weights (one model)
    [[nodiscard]] static std::vector<float> eval_host(std::span<weights_t const> weights,
                                                      std::span<std::uint64_t const> seeds, std::uint32_t max_moves) {
        std::vector<float> out(seeds.size());
        if (weights.size() < TA3B_NUM_PARAMS)
            throw std::runtime_error("ta3b: eval_host: weights.size() must be at least NUM_PARAMS");
        if (ta3b_eval_host(weights.data(), static_cast<std::uint32_t>(weights.size()), seeds.data(),
                           static_cast<std::uint32_t>(seeds.size()), max_moves, out.data(), nullptr,
                           nullptr) != TA3B_OK)
            throw std::runtime_error("ta3b: eval_host: invalid arguments");
        return out;
    }

    // extension: scores plus piece and line counts in one call
    void eval_full(std::span<weights_t const> weights, std::uint32_t num_models, std::span<std::uint64_t const> seeds,
                   std::uint32_t max_moves, std::vector<float>& score, std::vector<std::uint32_t>& pieces,
                   std::vector<std::uint32_t>& lines) {
        std::size_t const n = static_cast<std::size_t>(num_models) * seeds.size();
        score.resize(n);
        pieces.resize(n);
        lines.resize(n);
        check(ta3b_eval(_ctx.get(), weights.data(), num_models, static_cast<std::uint32_t>(
                            num_models ? weights.size() / num_models : TA3B_NUM_PARAMS),
                        seeds.data(), static_cast<std::uint32_t>(seeds.size()), max_moves, score.data(),
                        pieces.data(), lines.data()));
    }

private:
    void check(int rc) const {
        if (rc != TA3B_OK) throw std::runtime_error(std::string("ta3b: ") + ta3b_last_error(_ctx.get()));
    }
    struct Deleter {
        void operator()(ta3b_ctx* c) const { ta3b_destroy(c); }
    };
    std::unique_ptr<ta3b_ctx, Deleter> _ctx;
};

// model_eval.hpp:84-103: games seeds drawn from xoshiro256**(seed), shared by every model
inline std::vector<float> simulate(ModelEvaluator& evaluator, std::span<weights_t const> model_weights,
                                   std::size_t num_models, std::size_t games, std::uint64_t seed,
                                   std::size_t max_moves) {
    std::vector<std::uint64_t> seeds(games);
    ta3b_simulate_seeds(seed, static_cast<std::uint32_t>(games), seeds.data());
    return evaluator.eval(model_weights, static_cast<std::uint32_t>(num_models), seeds,
                          static_cast<std::uint32_t>(max_moves));
}

inline std::vector<float> simulate(ModelEvaluator& evaluator, std::span<weights_t const> model_weights,
                                   std::size_t games, std::uint64_t seed, std::size_t max_moves) {
    return simulate(evaluator, model_weights, 1, games, seed, max_moves);
}

} // namespace ta3::gpu
