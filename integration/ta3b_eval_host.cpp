// Caller-side CPU parity path: the definition of ta3b_eval_host (include/ta3b_host_ref.h),
// which include/ta3b.hpp's ta3::gpu::ModelEvaluator::eval_host forwards to.
//
// A trainer compiles this file into ITS OWN binary, in the place of the reference's
// ta3_gpu/src/common/model_eval_host.cpp, with the reference's headers on the include path
// (ta3_sim/incl, ta3_ai/incl, ta3_gpu/incl) and the same flags (C++23, no FP contraction).
// libta3b.so does not contain it: the evaluator library ships no CPU search, so there is no
// CPU fallback behind the GPU path; this is only the start-up self-check's other side
// (ta3_trainer/src/trainer2.cpp:57-89).
//
// The loop is the reference's game loop (model_eval_host.cpp:35-51): play up to max_moves
// moves with search_move_beam until the engine tops out, holding first when the chosen move
// says so, and feed stats_v4 after every placed piece; a game with no placed piece scores -1e6.
#include "ta3b_host_ref.h"

#include <ta3/gpu/detail/value_model.hpp>

#include <ta3/ai/models/metrics/tetris_stats_v4.hpp>
#include <ta3/ai/search/beam.hpp>
#include <ta3/sim/tetris_engine.hpp>

#include <cstddef>
#include <cstdint>

extern "C" int ta3b_eval_host(float const* weights, std::uint32_t num_params, std::uint64_t const* seeds,
                              std::uint32_t num_games, std::uint32_t max_moves, float* score_out,
                              std::uint32_t* pieces_out, std::uint32_t* lines_out) {
    namespace ai = ta3::ai;
    namespace sim = ta3::sim;
    constexpr std::size_t P = ai::model_t::NUM_PARAMS;
    if(num_games == 0)
        return TA3B_OK;
    if(weights == nullptr || seeds == nullptr || score_out == nullptr || num_params < P)
        return TA3B_ERR_ARG;

    ta3::gpu::net_ref const model{ai::model_t::weights_t{weights, P}};
    for(std::uint32_t g = 0; g < num_games; ++g) {
        sim::TetrisEngine game{seeds[g]};
        ai::stats_v4 stats{};
        std::uint32_t lines = 0;
        for(std::uint32_t move = 0; move < max_moves && !game.gameOver(); ++move) {
            auto const r = ai::search::search_move_beam(game, model);
            if(r.none())
                break;
            if(r.move.hold)
                game.hold();
            auto const cleared = game.place(r.move.orientation, r.move.x);
            if(cleared == sim::TetrisEngine::DIED)
                break;
            lines += static_cast<std::uint32_t>(cleared);
            stats.advance(game.board(), static_cast<std::uint32_t>(cleared));
        }
        score_out[g] = stats.piecesPlaced() == 0 ? -1.0e6f : static_cast<float>(stats.score());
        if(pieces_out != nullptr)
            pieces_out[g] = stats.piecesPlaced();
        if(lines_out != nullptr)
            lines_out[g] = lines;
    }
    return TA3B_OK;
}
