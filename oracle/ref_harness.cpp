// Test infrastructure only: a C-ABI wrapper around the reference's OWN CPU path
// (ta3_gpu/src/common/model_eval_host.cpp and the header-only ta3_sim / ta3_ai
// code it includes), compiled in place from the reference tree by
// oracle/Makefile into oracle/_ref/libta3ref.so.
//
// It is used for three things and nothing else:
//   * generating the golden vectors under tests/golden/ (gen_golden.py),
//   * pinning the C restatement in oracle/ta3_oracle.c against the reference,
//   * the reference arm / cpu_baseline of bench.py (timed CPU throughput).
// The product (tetris_ai3_b200) never loads this library.
#include "ta3/gpu/model_eval.hpp"
#include <ta3/gpu/detail/value_model.hpp>

#include <ta3/ai/search/beam.hpp>
#include <ta3/ai/models/metrics/tetris_stats_v4.hpp>
#include <ta3/sim/tetris_engine.hpp>

#include <atomic>
#include <random>
#include <cstdint>
#include <cstring>
#include <span>
#include <thread>
#include <vector>

namespace search = ta3::ai::search;
namespace sim = ta3::sim;
namespace ai = ta3::ai;

namespace {

constexpr std::size_t P = ai::model_t::NUM_PARAMS;

// net_ref plus a counter of value-model calls: one call == one evaluated
// beam placement, the unit of the throughput metric.
struct counting_ref {
    ta3::gpu::net_ref inner;
    std::uint64_t* counter;
    [[nodiscard]] constexpr search::value_t evaluate(search::clear_t c, sim::Board2 const& b, bool i) const {
        ++*counter;
        return inner.evaluate(c, b, i);
    }
};

struct game_out {
    float score;
    std::uint32_t pieces;
    std::uint32_t lines;
    std::uint64_t evals;
};

// The reference's customizable architecture widened: the v11 inputs
// (ModelV11::extractInputs, model_v11.hpp:63-91) through the reference's own
// dense layers (utility.hpp:29-46) 10 -> H ReLU -> H ReLU -> 1, weights of each
// layer as [out][in] then [out] biases: H = 64 gives 704 + 4160 + 65 = 4,929
// parameters, H = 32 gives 1,441.
template<std::size_t H>
struct wide_net {
    static constexpr std::size_t L1 = 10 * H + H, L2 = H * H + H, L3 = H + 1, P = L1 + L2 + L3;
};
constexpr std::size_t WIDE_H = 64;
constexpr std::size_t WIDE_P = wide_net<WIDE_H>::P;

template<std::size_t H>
struct counting_wide {
    using N = wide_net<H>;
    float const* w;
    std::uint64_t* counter;
    [[nodiscard]] search::value_t evaluate(search::clear_t c, sim::Board2 const& b, bool held_i) const {
        ++*counter;
        std::array<ai::data_t, ai::ModelV11::INPUTS> in{};
        ai::ModelV11::extractInputs(c, b, held_i, in);
        auto const h1 = ai::dense<10, H, true>(in, std::span<ai::data_t const, N::L1>{w, N::L1});
        auto const h2 = ai::dense<H, H, true>(h1, std::span<ai::data_t const, N::L2>{w + N::L1, N::L2});
        return ai::dense<H, 1, false>(h2, std::span<ai::data_t const, N::L3>{w + N::L1 + N::L2, N::L3})[0];
    }
};

// The loop of ModelEvaluator::eval_host (model_eval_host.cpp:35-51), with the
// piece / line counts and an optional per-move trace recorded on the side.
template<class Model>
game_out play_with(Model const& model, std::uint64_t& evals, std::uint64_t seed, std::uint32_t max_moves,
                   std::uint8_t* trace, std::uint32_t* n_moves, std::uint32_t* board_out);

game_out play(float const* w, std::uint64_t seed, std::uint32_t max_moves, std::uint8_t* trace,
              std::uint32_t* n_moves, std::uint32_t* board_out) {
    std::uint64_t evals = 0;
    counting_ref const model{ta3::gpu::net_ref{ai::model_t::weights_t{w, P}}, &evals};
    return play_with(model, evals, seed, max_moves, trace, n_moves, board_out);
}

template<std::size_t H>
game_out play_wide_h(float const* w, std::uint64_t seed, std::uint32_t max_moves, std::uint8_t* trace,
                     std::uint32_t* n_moves, std::uint32_t* board_out) {
    std::uint64_t evals = 0;
    counting_wide<H> const model{w, &evals};
    return play_with(model, evals, seed, max_moves, trace, n_moves, board_out);
}

game_out play_wide(float const* w, std::uint64_t seed, std::uint32_t max_moves, std::uint8_t* trace,
                   std::uint32_t* n_moves, std::uint32_t* board_out) {
    return play_wide_h<WIDE_H>(w, seed, max_moves, trace, n_moves, board_out);
}

template<class Model>
game_out play_with(Model const& model, std::uint64_t& evals, std::uint64_t seed, std::uint32_t max_moves,
                   std::uint8_t* trace, std::uint32_t* n_moves, std::uint32_t* board_out) {
    sim::TetrisEngine game{seed};
    ai::stats_v4 stats{};
    std::uint32_t lines = 0, moves = 0;
    for(std::uint32_t i = 0; i < max_moves && !game.gameOver(); ++i) {
        auto const r = search::search_move_beam(game, model);
        if(r.none())
            break;
        if(trace != nullptr) {
            trace[3 * moves + 0] = r.move.hold ? 1 : 0;
            trace[3 * moves + 1] = static_cast<std::uint8_t>(*r.move.orientation);
            trace[3 * moves + 2] = static_cast<std::uint8_t>(r.move.x + 2);
        }
        ++moves;
        if(r.move.hold)
            game.hold();
        auto const cleared = game.place(r.move.orientation, r.move.x);
        if(cleared == sim::TetrisEngine::DIED)
            break;
        lines += static_cast<std::uint32_t>(cleared);
        stats.advance(game.board(), static_cast<std::uint32_t>(cleared));
    }
    if(n_moves != nullptr)
        *n_moves = moves;
    if(board_out != nullptr)
        for(std::size_t x = 0; x < sim::WIDTH; ++x)
            board_out[x] = game.board().raw_column(x);
    float const score = stats.piecesPlaced() == 0 ? -1.0e6f : static_cast<float>(stats.score());
    return {score, stats.piecesPlaced(), lines, evals};
}

} // namespace

extern "C" {

std::uint32_t ta3ref_num_params() { return static_cast<std::uint32_t>(P); }
std::uint32_t ta3ref_num_params_wide() { return static_cast<std::uint32_t>(WIDE_P); }

// One game of the widened 10 -> 64 -> 64 -> 1 model, with its trace.
int ta3ref_play_wide(float const* w, std::uint64_t seed, std::uint32_t max_moves, float* score, std::uint32_t* pieces,
                     std::uint32_t* lines, std::uint64_t* evals, std::uint8_t* trace, std::uint32_t* n_moves,
                     std::uint32_t* board_out) {
    auto const r = play_wide(w, seed, max_moves, trace, n_moves, board_out);
    *score = r.score;
    *pieces = r.pieces;
    *lines = r.lines;
    *evals = r.evals;
    return 0;
}

// ModelEvaluator::eval_host itself, once per model (model-major output).
int ta3ref_eval_host(float const* w, std::uint32_t num_models, std::uint64_t const* seeds, std::uint32_t num_games,
                     std::uint32_t max_moves, float* score_out) {
    for(std::uint32_t m = 0; m < num_models; ++m) {
        auto const out = ta3::gpu::ModelEvaluator::eval_host(
            std::span<float const>{w + static_cast<std::size_t>(m) * P, P},
            std::span<std::uint64_t const>{seeds, num_games}, max_moves);
        std::memcpy(score_out + static_cast<std::size_t>(m) * num_games, out.data(), num_games * sizeof(float));
    }
    return 0;
}

// One game with its trace: trace gets 3 bytes per move (hold, orientation, x+2),
// capacity max_moves; board_out gets the final 10 bit-columns.
int ta3ref_play(float const* w, std::uint64_t seed, std::uint32_t max_moves, float* score, std::uint32_t* pieces,
                std::uint32_t* lines, std::uint64_t* evals, std::uint8_t* trace, std::uint32_t* n_moves,
                std::uint32_t* board_out) {
    auto const r = play(w, seed, max_moves, trace, n_moves, board_out);
    *score = r.score;
    *pieces = r.pieces;
    *lines = r.lines;
    *evals = r.evals;
    return 0;
}

// Multi-threaded batch over (model, game) pairs, pulled from an atomic ticket;
// the CPU baseline. Returns wall-clock-free results; the caller times it.
} // extern "C"

namespace {
using play_fn = game_out (*)(float const*, std::uint64_t, std::uint32_t, std::uint8_t*, std::uint32_t*,
                             std::uint32_t*);

int eval_mt(play_fn fn, std::size_t stride, float const* w, std::uint32_t num_models, std::uint64_t const* seeds,
            std::uint32_t num_games, std::uint32_t max_moves, std::uint32_t threads, float* score_out,
            std::uint32_t* pieces_out, std::uint32_t* lines_out, std::uint64_t* evals_total) {
    std::uint64_t const total = static_cast<std::uint64_t>(num_models) * num_games;
    std::atomic<std::uint64_t> next{0};
    std::atomic<std::uint64_t> evals{0};
    auto worker = [&] {
        std::uint64_t local = 0;
        for(;;) {
            auto const i = next.fetch_add(1);
            if(i >= total)
                break;
            auto const m = i / num_games, g = i % num_games;
            auto const r = fn(w + m * stride, seeds[g], max_moves, nullptr, nullptr, nullptr);
            score_out[i] = r.score;
            if(pieces_out)
                pieces_out[i] = r.pieces;
            if(lines_out)
                lines_out[i] = r.lines;
            local += r.evals;
        }
        evals += local;
    };
    if(threads <= 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for(std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back(worker);
        for(auto& t : pool)
            t.join();
    }
    if(evals_total)
        *evals_total = evals.load();
    return 0;
}
} // namespace

extern "C" {

int ta3ref_eval_mt(float const* w, std::uint32_t num_models, std::uint64_t const* seeds, std::uint32_t num_games,
                   std::uint32_t max_moves, std::uint32_t threads, float* score_out, std::uint32_t* pieces_out,
                   std::uint32_t* lines_out, std::uint64_t* evals_total) {
    return eval_mt(play, P, w, num_models, seeds, num_games, max_moves, threads, score_out, pieces_out, lines_out,
                   evals_total);
}

// the same batch for the widened 10 -> 64 -> 64 -> 1 model (4,929 parameters per model)
int ta3ref_eval_wide_mt(float const* w, std::uint32_t num_models, std::uint64_t const* seeds, std::uint32_t num_games,
                        std::uint32_t max_moves, std::uint32_t threads, float* score_out, std::uint32_t* pieces_out,
                        std::uint32_t* lines_out, std::uint64_t* evals_total) {
    return eval_mt(play_wide, WIDE_P, w, num_models, seeds, num_games, max_moves, threads, score_out, pieces_out,
                   lines_out, evals_total);
}

// the same batch for the 10 -> 32 -> 32 -> 1 model (1,441 parameters per model)
int ta3ref_eval_wide32_mt(float const* w, std::uint32_t num_models, std::uint64_t const* seeds,
                          std::uint32_t num_games, std::uint32_t max_moves, std::uint32_t threads, float* score_out,
                          std::uint32_t* pieces_out, std::uint32_t* lines_out, std::uint64_t* evals_total) {
    return eval_mt(play_wide_h<32>, wide_net<32>::P, w, num_models, seeds, num_games, max_moves, threads, score_out,
                   pieces_out, lines_out, evals_total);
}

// Weights of ta3_gpu/tests/src/parity_test.cpp:20-32: mt19937{seed} with
// uniform_real_distribution<float> over the model bounds [-2, 2].
void ta3ref_parity_weights(std::uint32_t seed, float* out) {
    std::mt19937 rng{seed};
    auto const bounds = ai::model_t::bounds();
    std::uniform_real_distribution<float> dist{static_cast<float>(bounds.x), static_cast<float>(bounds.y)};
    for(std::size_t i = 0; i < P; ++i)
        out[i] = dist(rng);
}

// Weights of the trainer's start-up parity self-check, ta3_trainer/src/trainer2.cpp:58-67 (2 models).
void ta3ref_selfcheck_weights(float* out2p) {
    sim::xoshiro256ss rng{0xC0FFEEull};
    for(std::size_t i = 0; i < 2 * P; ++i)
        out2p[i] = static_cast<float>(ai::m::BOUNDS[0]
            + (ai::m::BOUNDS[1] - ai::m::BOUNDS[0]) * (static_cast<double>(rng() >> 11) * 0x1.0p-53));
}

// The gpu::simulate seed derivation (model_eval.hpp:148-151).
void ta3ref_simulate_seeds(std::uint64_t seed, std::uint32_t games, std::uint64_t* out) {
    sim::xoshiro256ss gen{seed};
    for(std::uint32_t i = 0; i < games; ++i)
        out[i] = gen();
}

// Piece sequence of a fresh engine: current piece after each of n plain placements
// is not observable without placing, so expose the raw bag draw order instead.
void ta3ref_piece_queue(std::uint64_t seed, std::uint32_t* queue6) {
    sim::TetrisEngine const game{seed};
    queue6[0] = *game.currentPiece();
    for(std::size_t i = 0; i < 5; ++i)
        queue6[1 + i] = *game.lookahead()[i];
}

// Placement LUT: for piece p, count and (orientation, x) per index.
std::uint32_t ta3ref_placements(std::uint32_t piece, std::uint8_t* orient, std::int8_t* x, std::uint16_t* cols,
                                std::int8_t* col0) {
    auto const pt = static_cast<sim::PieceType>(piece);
    auto const n = search::n_theoretical_placements(pt);
    for(std::uint32_t i = 0; i < n; ++i) {
        auto const pl = search::nth_placement(pt, i);
        orient[i] = static_cast<std::uint8_t>(*pl.orientation);
        x[i] = static_cast<std::int8_t>(pl.x);
        cols[i] = pl.shape.cols;
        col0[i] = static_cast<std::int8_t>(pl.shape.col0);
    }
    return n;
}

// Plan tree dump: per layer, count and per node (slot, parent, childBegin, childEnd, rootHold, heldSlot).
void ta3ref_plan_tree(std::uint32_t held_empty, std::uint32_t* counts, std::uint8_t* nodes6) {
    auto const& tree = search::dev::PLAN_TREES[held_empty ? 1 : 0];
    for(std::uint32_t l = 0; l < search::DEPTH; ++l) {
        counts[l] = tree.count[l];
        for(std::uint32_t n = 0; n < search::MAX_SEQUENCES; ++n) {
            auto const& node = tree.nodes[l][n];
            auto* o = nodes6 + (l * search::MAX_SEQUENCES + n) * 6;
            o[0] = node.slot;
            o[1] = node.parentIdx;
            o[2] = node.childBegin;
            o[3] = node.childEnd;
            o[4] = node.rootHold ? 1 : 0;
            o[5] = node.heldSlot;
        }
    }
}

void ta3ref_search_consts(std::uint32_t* out) {
    out[0] = search::DEPTH;
    out[1] = search::MAX_PLACEMENTS;
    out[2] = search::MAX_ROOT_GROUPS;
    out[3] = search::MAX_CHILD_MID;
    out[4] = search::MAX_LAST;
    out[5] = search::ROOT_SLOTS;
    out[6] = search::mid_slots(search::BEAM_WIDTHS);
    out[7] = search::leaf_orders(search::last_width(search::BEAM_WIDTHS));
    out[8] = search::order_span(search::BEAM_WIDTHS);
}

// Value model features and output for one board (ModelV11::extractInputs / evaluate).
float ta3ref_evaluate(float const* w, std::uint32_t const* cols10, std::uint32_t clear_bits, int held_is_i,
                      float* features10) {
    sim::Board2 board{};
    // rebuild the board from raw columns: place single cells via the one-cell shape
    for(std::size_t x = 0; x < sim::WIDTH; ++x)
        for(std::uint32_t y = 0; y < sim::HEIGHT; ++y)
            if((cols10[x] >> y) & 1u)
                board.place(sim::piece_shape{1, static_cast<int>(x)}, static_cast<int>(y));
    std::array<float, ai::model_t::INPUTS> in{};
    ai::model_t::extractInputs(ai::clear_hist_t{clear_bits}, board, held_is_i != 0, in);
    for(std::size_t i = 0; i < in.size(); ++i)
        features10[i] = in[i];
    return ai::model_t::evaluate(ai::clear_hist_t{clear_bits}, board, held_is_i != 0, ai::model_t::weights_t{w, P});
}

// Apply one placement to a board the way the search does (search.hpp:61-70).
int ta3ref_apply(std::uint32_t const* cols10, std::uint32_t piece, std::uint32_t index, std::uint32_t* out10,
                 std::uint32_t* cleared) {
    sim::Board2 board{};
    for(std::size_t x = 0; x < sim::WIDTH; ++x)
        for(std::uint32_t y = 0; y < sim::HEIGHT; ++y)
            if((cols10[x] >> y) & 1u)
                board.place(sim::piece_shape{1, static_cast<int>(x)}, static_cast<int>(y));
    auto const s = search::apply(board, {}, search::nth_placement(static_cast<sim::PieceType>(piece), index));
    for(std::size_t x = 0; x < sim::WIDTH; ++x)
        out10[x] = s.nextBoard.raw_column(x);
    *cleared = s.nextClearHist.lines();
    return s.legal ? 1 : 0;
}

} // extern "C"
