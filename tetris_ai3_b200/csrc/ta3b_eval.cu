// B200 (sm_100a) model x game beam-search evaluator: kernel and C ABI.
//
// One warp plays one (model, game) sim from reset to the move cap or top-out;
// a persistent grid pulls sims from a device ticket counter, so warps that
// finish short games immediately start new ones (sims are very uneven: bad
// weights top out in tens of pieces, good ones play to the cap).
//
// Per move (the reference's search_move_beam, ta3_ai/incl/ta3/ai/search/beam.hpp:484-570):
//   root stage    <= 68 candidates  -> top 16          (beam.hpp:283-301, 507-513)
//   mid level 1   <= 1088           -> top 32          (beam.hpp:337-403)
//   mid level 2   <= 2176           -> top 32
//   leaf stage    <= 2176           -> argmax key      (beam.hpp:407-443)
// Lanes stride the flattened (parent, child list, placement) space of a level.
// Each kept frontier node gets a parent record in shared memory (heights,
// holes, row fills, feature totals, hidden-layer partial sums; eval_core.h),
// so a candidate is evaluated incrementally from the <= 4 columns it touches;
// candidates that clear a row or reach into the spawn rows are queued and
// evaluated by the full reference algorithm in compacted 32-lane batches.
// The top-K of a level is a warp-distributed sorted list (lane i holds the
// i-th best packed key) maintained with ballots and shuffles, so level scores
// never touch memory. Nothing in the move loop synchronises more than one warp.
#include "ta3b.h"
#include "tables.h"
#include "eval_core.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace ta3b {
namespace {

constexpr int WARP = 32;
constexpr uint32_t FULL_MASK = 0xFFFFFFFFu;
// The work queue's scratch words: a 64-bit sim ticket (words 0-1) and the error status (word 2:
// bit 0 = a search found no move although a root was legal, bit 1 = the time budget ran out).
constexpr int kStatusWord = 2;
// the tail hand-off (single-warp kernel -> paired kernel): warps that found no sim, the hand-off
// flag, games checkpointed, and the paired kernel's ticket over the checkpoints
constexpr int kDoneWord = 3, kHandoffWord = 4, kCkptCountWord = 5, kCkptTicketWord = 6;
constexpr size_t kScratchBytes = 32;
constexpr uint32_t kNoSim = 0xFFFFFFFFu;                 // never a sim index: sims <= 2^32 - 1
constexpr uint64_t kMaxSims = 0xFFFFFFFFull;

// ---------------------------------------------------------------- tables ---
struct DevTables {
    uint32_t nplace[NPIECE];
    uint32_t spawn_cols[NPIECE];
    uint32_t spawn_col0[NPIECE];
    uint32_t shape_cols[NPIECE][4];
    int32_t shape_left[NPIECE][4];
    // per tree [held_empty][layer][node]: slot | held << 4 | root_hold << 8
    uint32_t node[2][DEPTH][16];
};

constexpr DevTables make_dev_tables() {
    DevTables d{};
    for (int p = 0; p < NPIECE; ++p) {
        d.nplace[p] = TABLES.nplace[p];
        d.spawn_cols[p] = TABLES.spawn_cols[p];
        d.spawn_col0[p] = uint32_t(TABLES.spawn_col0[p]);
        for (int o = 0; o < 4; ++o) {
            d.shape_cols[p][o] = TABLES.shape_cols[p][o];
            d.shape_left[p][o] = TABLES.shape_left[p][o];
        }
    }
    for (int he = 0; he < 2; ++he)
        for (int l = 0; l < DEPTH; ++l)
            for (int n = 0; n < 16; ++n) {
                TreeNode const& t = TABLES.tree[he][l][n];
                d.node[he][l][n] = uint32_t(t.slot) | (uint32_t(t.held) << 4) | (uint32_t(t.root_hold) << 8);
            }
    return d;
}

__constant__ DevTables c_tables = make_dev_tables();

// Placement tables copied into shared memory per block: the incremental-path
// data (PlaceFast) and the move itself packed as cols (16) | col0 (4) << 16 |
// orientation (2) << 20 | (x + 2) (4) << 24.
struct LutTables {
    PlaceFast fast[NPIECE][MP];
    uint32_t move[NPIECE][MP];
};
constexpr LutTables make_lut_tables() {
    LutTables t{};
    for (int p = 0; p < NPIECE; ++p)
        for (int i = 0; i < TABLES.nplace[p]; ++i) {
            Place const pl = TABLES.place[p][i];
            t.fast[p][i] = FAST.place[p][i];
            t.move[p][i] = uint32_t(pl.cols) | (uint32_t(pl.col0) << 16) | (uint32_t(pl.orient) << 20) |
                           (uint32_t(pl.x + 2) << 24);
        }
    return t;
}
__device__ LutTables const g_lut = make_lut_tables();

__device__ __forceinline__ float ordered_bits_inv(uint32_t s) {              // beam.hpp:209-211
    return __uint_as_float((s & 0x80000000u) ? (s ^ 0x80000000u) : ~s);
}

// ------------------------------------------------------------ game state ---
struct Engine {                      // ta3_sim/incl/ta3/sim/tetris_engine.hpp:101-163
    uint32_t board[12];              // 10 bit-columns, padded to 48 bytes for 16-byte loads
    uint64_t rng[4];
    uint32_t queue[QUEUE];
    uint32_t bag[7];
    uint32_t bag_pos;
    uint32_t held;
    uint32_t over;
};

struct Stats {                       // the stats_v4 fields score_v1 reads
    uint32_t pieces, lines;
    uint32_t clears[5];
    uint32_t sum_max_height;
    uint32_t sum_hole_depths;
};

__device__ uint64_t rng_next(uint64_t (&s)[4]) {                             // xoshiro256ss.hpp:33-45
    uint64_t const res = ((s[1] * 5) << 7 | (s[1] * 5) >> 57) * 9;
    uint64_t const t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return res;
}

__device__ uint32_t draw_piece(Engine& e) {                                  // tetris_engine.hpp:116-129
    if (e.bag_pos > 0) return e.bag[--e.bag_pos];
    for (int i = 0; i < 7; ++i) e.bag[i] = uint32_t(i);
    for (uint32_t i = 6; i > 0; --i) {
        uint32_t const j = uint32_t(rng_next(e.rng) % uint64_t(i + 1));
        uint32_t const t = e.bag[i];
        e.bag[i] = e.bag[j];
        e.bag[j] = t;
    }
    e.bag_pos = 6;
    return e.bag[6];
}

__device__ void update_game_over(Engine& e) {                                // tetris_engine.hpp:159-161
    uint32_t const p = e.queue[0];
    uint32_t const cols = c_tables.spawn_cols[p];
    int const col0 = int(c_tables.spawn_col0[p]);
    uint32_t hit = 0;
    for (int i = 0; i < 4; ++i) {
        int const x = col0 + i;
        if (x < W) hit |= e.board[x] & ((cols >> (4 * i)) & 0xFu);
    }
    e.over = hit != 0;
}

__device__ void engine_reset(Engine& e, uint64_t seed) {                     // tetris_engine.hpp:103-114
    for (int x = 0; x < 12; ++x) e.board[x] = 0;
    for (int i = 0; i < 4; ++i) {                                            // xoshiro256ss.hpp:20-28
        seed += 0x9e3779b97f4a7c15ULL;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        e.rng[i] = z ^ (z >> 31);
    }
    e.held = NO_PIECE;
    e.bag_pos = 0;
    for (int i = 0; i < QUEUE; ++i) e.queue[i] = draw_piece(e);
    update_game_over(e);
}

__device__ void advance_queue(Engine& e) {                                   // tetris_engine.hpp:131-135
    for (int i = 1; i < QUEUE; ++i) e.queue[i - 1] = e.queue[i];
    e.queue[QUEUE - 1] = draw_piece(e);
}

__device__ void engine_hold(Engine& e) {                                     // tetris_engine.hpp:148-157
    if (e.held == NO_PIECE) {
        e.held = e.queue[0];
        advance_queue(e);
    } else {
        uint32_t const t = e.held;
        e.held = e.queue[0];
        e.queue[0] = t;
    }
    update_game_over(e);
}

__device__ __forceinline__ void load_board(uint32_t const* __restrict__ src, uint32_t (&b)[W]);

// The drop + lock + clear of one placement (search.hpp:61-70, board2.hpp:306-342) and the
// integer metrics of the resulting board (v_board_metrics.hpp:130-225): one body for the
// deferred candidates' full path and the engine's commit, so the kernel holds one copy of
// it. src is 16-byte aligned; dst (may be null, may equal src) receives the new board.
struct Applied {
    BoardInts bi;
    int cleared;
    bool legal;
};
__device__ __noinline__ Applied apply_ints(uint32_t const* src, uint32_t cols, int col0, uint32_t* dst) {
    uint32_t b[W], nb[W];
    load_board(src, b);
    Applied r{};
    r.legal = apply_full(b, cols, col0, nb, r.cleared);
    if (!r.legal) return r;
    r.bi = board_ints(nb);
    if (dst)
        for (int c = 0; c < W; ++c) dst[c] = nb[c];
    return r;
}

// hard drop at window x-origin x in orientation o; returns rows cleared or -1 on top-out,
// and the new board's metrics in bi
__device__ int engine_place(Engine& e, int o, int x, BoardInts& bi) {         // tetris_engine.hpp:137-146
    uint32_t const p = e.queue[0];
    uint32_t const cols = c_tables.shape_cols[p][o];
    int const col0 = x + c_tables.shape_left[p][o];
    // the search only commits legal moves, so this is the drop + lock + clear of board2.hpp
    Applied const a = apply_ints(e.board, cols, col0, e.board);
    bi = a.bi;
    advance_queue(e);
    update_game_over(e);
    return e.over ? -1 : a.cleared;
}

// ------------------------------------------------------------ candidates ---
struct SmemW {                       // weights read from shared memory (broadcast loads)
    static constexpr bool VEC4 = false;
    float const* p;
    __device__ __forceinline__ float operator()(int i) const { return p[i]; }
};
struct GlobalW {
    static constexpr bool VEC4 = false;
    float const* p;
    __device__ __forceinline__ float operator()(int i) const { return __ldg(p + i); }
};
__device__ __forceinline__ void load_board(uint32_t const* __restrict__ src, uint32_t (&b)[W]) {
    uint4 const q0 = *reinterpret_cast<uint4 const*>(src);
    uint4 const q1 = *reinterpret_cast<uint4 const*>(src + 4);
    uint2 const q2 = *reinterpret_cast<uint2 const*>(src + 8);
    b[0] = q0.x; b[1] = q0.y; b[2] = q0.z; b[3] = q0.w;
    b[4] = q1.x; b[5] = q1.y; b[6] = q1.z; b[7] = q1.w;
    b[8] = q2.x; b[9] = q2.y;
}

#ifndef TA3B_MLP_MODE
#define TA3B_MLP_MODE MLP_X2MUL     // packed multiplies, scalar adds: the reference's roundings, fewer instructions
#endif

// fast path: read the parent-record words this placement needs, then eval_core's fast_eval
template <int MLP = TA3B_MLP_MODE>
__device__ __forceinline__ int fast_candidate(uint32_t const* __restrict__ rec, PlaceFast pf, bool held_i,
                                              FastW const& fw, float& v, float* dbg = nullptr) {
    RecView r;
    float4 const p0 = *reinterpret_cast<float4 const*>(rec + R_P);
    float4 const p1 = *reinterpret_cast<float4 const*>(rec + R_P + 4);
    r.P[0] = p0.x; r.P[1] = p0.y; r.P[2] = p0.z; r.P[3] = p0.w;
    r.P[4] = p1.x; r.P[5] = p1.y; r.P[6] = p1.z; r.P[7] = p1.w;
    uint4 const q = *reinterpret_cast<uint4 const*>(rec + R_HD);       // hd, rc0, rc1, rc2
    r.hd = q.x; r.rc0 = q.y; r.rc1 = q.z; r.rc2 = q.w;
    r.tot = rec[R_TOT];
    span_of(rec, int((pf.m >> 27) & 0xFu), r.h4, r.hm4);
    r.combo = rec[R_COMBO + ((pf.m >> 16) & 63u)];
    return fast_eval<MLP>(r, pf, held_i, fw, v, dbg);
}

// ------------------------------------------------ widened network (device) ---
// One lane = one candidate; the warp's lanes run the network together so that a
// term can be left out when its input is exactly zero in every lane. That is
// exact: x + (±0 * w) == x for finite w and every x but -0, and a sum that starts
// from a bias other than -0 is never -0 (under round-to-nearest a sum is -0 only
// for (-0) + (-0)). repack_wide_kernel sets WIDE_SKIP for models whose weights
// are all finite and whose biases are not -0; every other model runs every term.
// Each unit's sum keeps the reference order (utility.hpp:30-46: bias, then the
// inputs ascending), only without the zero terms. Lanes without a candidate pass
// zero inputs. hb: this warp's hidden-unit buffer, [unit][lane] floats (no bank conflicts).
struct WideIn {
    float v[NIN];
};
template <int H>
constexpr int kWideHbFloats = H * WARP;                // per warp: H units x 32 lanes (8 KB for 64)

// four units' sums += x * q: the products as two packed multiplies (each half rounded like the
// scalar multiply), the additions scalar, so that no multiply is fused into an add
__device__ __forceinline__ void wide_fold4(float* a, float2 x, float4 q) {
    float2 const p01 = f2_mul(x, make_float2(q.x, q.y));
    float2 const p23 = f2_mul(x, make_float2(q.z, q.w));
    a[0] = f_add(a[0], p01.x);
    a[1] = f_add(a[1], p01.y);
    a[2] = f_add(a[2], p23.x);
    a[3] = f_add(a[3], p23.y);
}

template <int H>
__device__ __noinline__ float wide_value(WideIn in, float const* __restrict__ w, float* __restrict__ hb, int lane) {
    static_assert(H >= 4 && H <= 64 && H % 4 == 0, "the hidden-unit masks hold 64 units");
    using D = WideNet<H>;
    uint32_t const skip = __ldg(reinterpret_cast<uint32_t const*>(w) + D::SKIP);
    float a[H];
#pragma unroll
    for (int o = 0; o < H; o += 4) {
        float4 const b = __ldg(reinterpret_cast<float4 const*>(w + D::B1 + o));
        a[o] = b.x; a[o + 1] = b.y; a[o + 2] = b.z; a[o + 3] = b.w;
    }
    // layer 1, one input at a time over all 64 units (inputs that are zero in every lane skipped)
    uint32_t inz = 0;
#pragma unroll
    for (int i = 0; i < NIN; ++i) inz |= in.v[i] != 0.0f ? 1u << i : 0u;
    inz = skip ? __reduce_or_sync(FULL_MASK, inz) : (1u << NIN) - 1u;
#pragma unroll
    for (int i = 0; i < NIN; ++i) {
        if (!((inz >> i) & 1u)) continue;
        float4 const* wr = reinterpret_cast<float4 const*>(w + D::W1T + i * H);
        float2 const x = make_float2(in.v[i], in.v[i]);
#pragma unroll
        for (int o = 0; o < H; o += 4) {
            float4 const q = __ldg(wr + o / 4);
            wide_fold4(a + o, x, q);
        }
    }
    // ReLU into the buffer; nz = the units that are non-zero in some lane
    uint32_t nz[2] = {0u, 0u};
#pragma unroll
    for (int o = 0; o < H; o += 4) {
        float4 const h = make_float4(relu(a[o]), relu(a[o + 1]), relu(a[o + 2]), relu(a[o + 3]));
        float* const hq = hb + lane;
        hq[(o + 0) * WARP] = h.x;
        hq[(o + 1) * WARP] = h.y;
        hq[(o + 2) * WARP] = h.z;
        hq[(o + 3) * WARP] = h.w;
        uint32_t const bits = (h.x != 0.0f ? 1u : 0u) | (h.y != 0.0f ? 2u : 0u) | (h.z != 0.0f ? 4u : 0u) |
                              (h.w != 0.0f ? 8u : 0u);
        nz[o >> 5] |= bits << (o & 31);
    }
    if (skip) {
        nz[0] = __reduce_or_sync(FULL_MASK, nz[0]);
        nz[1] = __reduce_or_sync(FULL_MASK, nz[1]);
    } else {
        nz[0] = nz[1] = ~0u;
    }
    // layer 2, one hidden unit at a time over all 64 outputs
#pragma unroll
    for (int o = 0; o < H; o += 4) {
        float4 const b = __ldg(reinterpret_cast<float4 const*>(w + D::B2 + o));
        a[o] = b.x; a[o + 1] = b.y; a[o + 2] = b.z; a[o + 3] = b.w;
    }
    float const* hs = hb + lane;
    uint64_t m = (uint64_t(nz[1]) << 32) | nz[0];
    if (H < 64) m &= (uint64_t(1) << (H & 63)) - 1u;         // only the H units that exist
    while (m) {
        int const i = __ffsll(static_cast<long long>(m)) - 1;
        m &= m - 1;
        float2 const x = make_float2(hs[i * WARP], hs[i * WARP]);
        float4 const* wr = reinterpret_cast<float4 const*>(w + D::W2T + i * H);
#pragma unroll
        for (int o = 0; o < H; o += 4) {
            float4 const q = __ldg(wr + o / 4);
            wide_fold4(a + o, x, q);
        }
    }
    // layer 3: every term, ascending
    float out = __ldg(w + D::B3);
#pragma unroll
    for (int o = 0; o < H; o += 4) {
        float4 const q = __ldg(reinterpret_cast<float4 const*>(w + D::W3 + o));
        float2 const t01 = f2_mul(make_float2(relu(a[o]), relu(a[o + 1])), make_float2(q.x, q.y));
        float2 const t23 = f2_mul(make_float2(relu(a[o + 2]), relu(a[o + 3])), make_float2(q.z, q.w));
        out = f_add(out, t01.x);
        out = f_add(out, t01.y);
        out = f_add(out, t23.x);
        out = f_add(out, t23.y);
    }
    return out;
}

// fast path of the widened network: the same record words; every lane of the warp calls it
template <int H>
__device__ __forceinline__ int fast_candidate_wide(uint32_t const* __restrict__ rec, PlaceFast pf, bool held_i,
                                                   float const* __restrict__ w, float* hb, int lane, float& v) {
    RecView r;
    uint4 const q = *reinterpret_cast<uint4 const*>(rec + R_HD);
    r.hd = q.x; r.rc0 = q.y; r.rc1 = q.z; r.rc2 = q.w;
    r.tot = rec[R_TOT];
    span_of(rec, int((pf.m >> 27) & 0xFu), r.h4, r.hm4);
    r.combo = rec[R_COMBO + ((pf.m >> 16) & 63u)];
    WideIn in;
    bool const defer = fast_wide_inputs(r, rec[R_CLEARS], pf, held_i, in.v);
    v = wide_value<H>(in, w, hb, lane);
    return defer ? FAST_DEFER : FAST_OK;
}

// stats_v4::advance (tetris_stats.hpp:19-23 with metrics.hpp:196-229); bi: the board's metrics
__device__ void stats_advance(Stats& st, BoardInts const& bi, uint32_t lines) {
    st.pieces += 1;
    st.lines += lines;
    st.clears[lines] += 1;
    st.sum_max_height += bi.max_height;
    st.sum_hole_depths += bi.hole_depths;
}

// score_v1 (ta3_ai/incl/ta3/ai/models/metrics/score_v1.hpp:8-34) in FP64, no contraction
__device__ float final_score(Stats const& st) {
    if (st.pieces == 0) return -1.0e6f;                                      // model_eval_host.cpp:51
    double const pay[5] = {0.0, 0.2, 0.8, 2.0, 10.0};
    double cb = 0.0;
    for (int k = 1; k < 5; ++k) cb = __dadd_rn(cb, __dmul_rn(pay[k], double(st.clears[k])));
    double const n = double(st.pieces);
    double const surv = __dmul_rn(0.02, n);
    double const avg_h = __ddiv_rn(double(st.sum_max_height), n);
    double const over = __dadd_rn(avg_h, -12.0);
    double const hpen = __dmul_rn(over < 0.0 ? 0.0 : over, 1.0);
    double const dpen = __dmul_rn(__ddiv_rn(double(st.sum_hole_depths), n), 1.5);
    return __double2float_rn(__dadd_rn(__dadd_rn(__dadd_rn(cb, surv), -hpen), -dpen));
}

// ------------------------------------------------------------------ top-K ---
__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    return (uint64_t(__shfl_sync(FULL_MASK, uint32_t(v >> 32), src)) << 32) | __shfl_sync(FULL_MASK, uint32_t(v), src);
}
__device__ __forceinline__ uint64_t shfl64_up(uint64_t v) {
    return (uint64_t(__shfl_up_sync(FULL_MASK, uint32_t(v >> 32), 1)) << 32) | __shfl_up_sync(FULL_MASK, uint32_t(v), 1);
}

__device__ __forceinline__ uint64_t shfl64_xor(uint64_t v, int m) {
    return (uint64_t(__shfl_xor_sync(FULL_MASK, uint32_t(v >> 32), m)) << 32) | __shfl_xor_sync(FULL_MASK, uint32_t(v), m);
}

// Bitonic sort of one key per lane into descending order (lane i = i-th largest).
__device__ __forceinline__ uint64_t warp_sort_desc(uint64_t v, int lane) {
#pragma unroll
    for (int k = 2; k <= WARP; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            uint64_t const o = shfl64_xor(v, j);
            bool const keep_max = ((lane & j) == 0) == ((lane & k) == 0);   // descending runs where lane & k == 0
            v = keep_max ? (v > o ? v : o) : (v < o ? v : o);
        }
    }
    return v;
}

// Bitonic merge of two descending 32-key lists (lane i = i-th largest) into the top kl keys.
__device__ __forceinline__ uint64_t merge_topk(uint64_t a, uint64_t b, int kl, int lane) {
    uint64_t const rb = shfl64(b, 31 - lane);                    // ascending
    uint64_t c = a > rb ? a : rb;                                // bitonic, holds the 32 largest of both
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        uint64_t const o = shfl64_xor(c, j);
        bool const lower = (lane & j) == 0;
        c = lower ? (c > o ? c : o) : (c < o ? c : o);
    }
    return lane < kl ? c : 0ull;
}

// Fold one key per lane into the warp's sorted top-K list (lane i = i-th largest, 0 = empty;
// `thr` caches list[k-1]): the keys above thr are inserted one at a time by ballot/shuffle. The
// threshold is refreshed once per round, not after every insertion: a key that an earlier
// insertion of the same round pushed below the list finds its position >= k and changes nothing
// (3 % faster on the headline generation than refreshing and re-filtering per insertion).
__device__ __forceinline__ void topk_fold(uint64_t& list, uint64_t& thr, uint64_t key, int k, int lane) {
    uint32_t mask = __ballot_sync(FULL_MASK, key > thr);
    if (!mask) return;
    while (mask) {
        int const s = __ffs(int(mask)) - 1;
        uint64_t const x = shfl64(key, s);
        int const pos = __popc(__ballot_sync(FULL_MASK, list > x));
        uint64_t const up = shfl64_up(list);
        if (lane > pos && lane < k) list = up;
        if (lane == pos && pos < k) list = x;
        mask &= mask - 1u;
    }
    thr = shfl64(list, k - 1);
}

__device__ __forceinline__ uint64_t warp_max64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t const u = shfl64(v, int((threadIdx.x + o) & 31u));
        v = u > v ? u : v;
    }
    return v;
}

// ----------------------------------------------------------------- teams ---
// Team kernels play every game with TEAM (2, 4 or 8) consecutive warps of a block: the first
// warp (the leader) owns the game and runs everything but the candidate passes alone; in each
// stage the team's warps take the 32-candidate rounds in turn (warp r of the team takes rounds
// r, r + TEAM, r + 2 TEAM, ...), each keeps its own top-K list, argmax, legality bits and
// evaluation count, and the leader merges the partners' (keys are unique within a stage, so the
// result is the single-warp one). A game therefore runs faster while the issue work per move stays
// the same, which shortens a launch's tail of long games. A team synchronises through an mbarrier
// whose waits give up after kTeamWaitNs (no legitimate wait comes near it): the warp sets status
// bit STATUS_TEAM and leaves, and the call reports TA3B_ERR_DEVICE.
constexpr uint32_t TEAM_GAME_END = 0xFFFFFFFFu;
constexpr unsigned long long kTeamWaitNs = 1000000000ull;    // 1 s
constexpr uint32_t STATUS_TEAM = 4u;
// a partner's stage results, in its own (otherwise unused) record area: its list (or per-lane
// argmax) in words 0-63, its legality bits in words X_LO / X_HI; its game's evaluation count in
// X_EVALS
constexpr int X_LO = 64, X_HI = 65, X_EVALS = 66;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------- kernel ---
struct alignas(16) WarpShared {
    uint32_t rec[33][REC_WORDS];      // kept frontier records (rank -> record); [32] = committed board
    float wfull[NPARAMS + 3];         // the v11 model's weights (full path, record partial sums)
    float const* wglobal;              // the widened model's weights (global memory)
    unsigned long long t_start;        // the launch's start on this warp (time budget)
    Engine eng;                        // the committed game
    Stats st;
    uint32_t seg_off[65];              // a level's candidate segments (parent rank, child list)
    uint32_t seg_info[64];             // rec (6) | rank k << 8 | piece << 16 | held-is-I << 20 | child << 21
    uint32_t defer[64];                // queued (segment << 8 | placement) for the full path
    alignas(8) uint64_t kbuf[WARP];    // a level's keys above the top-K threshold, not yet merged
    // team kernels (TEAM warps per game; the game lives in the leader's area)
    alignas(8) unsigned long long team_bar;   // game area: the team's barrier (an mbarrier of TEAM arrivals)
    uint32_t team_cmd;                 // game area: the stage to run next, or TEAM_GAME_END
    uint32_t team_total;               // game area: that stage's candidate count
    uint32_t team_sim;                 // game area: the sim the team plays (kNoSim: none left)
    uint32_t team_broken;              // this warp: a team wait ran out
    uint32_t pad_team_[2];
};
static_assert(sizeof(WarpShared) % 16 == 0, "warp blocks must keep 16-byte alignment");

// The team barrier (pr[0] the leader's area, pr[r] warp r's): an mbarrier in the game area that
// completes a phase when every team warp's lane 0 has arrived. Arrival releases and the wait
// acquires, so the warps' shared-memory writes before the barrier are visible to the others after
// it. The wait polls mbarrier.try_wait (which suspends the thread in hardware between polls) and
// gives up after kTeamWaitNs: false = it ran out (status bit set, this warp's team_broken set).
__device__ __forceinline__ void team_bar_init(WarpShared* pr, uint32_t team) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 ::"r"(uint32_t(__cvta_generic_to_shared(&pr[0].team_bar))), "r"(team)
                 : "memory");
}

__device__ __forceinline__ bool team_sync(WarpShared* pr, int rank, uint32_t* status, int lane) {
    int ok = 1;
    __syncwarp();
    if (lane == 0) {
        uint32_t const bar = uint32_t(__cvta_generic_to_shared(&pr[0].team_bar));
        unsigned long long state;
        asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(bar) : "memory");
        unsigned long long t0 = 0;
        for (uint32_t polls = 0;; ++polls) {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(bar), "l"(state)
                : "memory");
            if (done) break;
            if (polls == 0) t0 = global_ns();
            else if ((polls & 15u) == 0 && global_ns() - t0 > kTeamWaitNs) {
                atomicOr(status, STATUS_TEAM);
                pr[rank].team_broken = 1u;
                ok = 0;
                break;
            }
        }
    }
    ok = __shfl_sync(FULL_MASK, ok, 0);
    __syncwarp();
    return ok != 0;
}

struct Params {
    float const* weights;
    uint64_t const* seeds;
    float* score;
    uint32_t* pieces;
    uint32_t* lines;
    uint32_t* evals;
    uint8_t* trace;
    uint32_t* n_moves;
    uint32_t* board_out;
    uint32_t* scratch;                 // 16-byte aligned: [0..1] 64-bit sim ticket, [2] error status,
                                       // [3..6] the tail hand-off's words
    unsigned long long* timing;        // optional: per sim [start, end] global timer (ns)
    unsigned long long* keys;          // tracing flavour: per move the final argmax's two largest keys
    unsigned long long budget_ns;      // 0, or the launch's time budget: past it warps stop and set status bit 2
    uint32_t num_games, models_per_island, max_moves, total_sims;
    uint32_t warps_active;             // 0, or the warps of each block that play (a batch smaller than
                                       // the grid's slots is spread over every SM); the rest take no sim
    struct Checkpoint* ckpt;           // the tail hand-off's checkpoints (ckpt_cap of them)
    uint32_t ckpt_cap;
    uint32_t handoff_at;               // hand-off flavour: hand the games over when at most this many play
    uint32_t resume;                   // paired kernel: play the checkpointed games instead of the sims
    uint32_t test_flags;               // tests only: bit 0 = team partners leave at launch start, so
                                       // the leaders' first team wait runs out (status bit 4)
};

// A game handed from the single-warp kernel to the paired kernel at a move boundary.
struct Checkpoint {
    Engine eng;
    Stats st;
    uint32_t sim, moves, evals, pad;
};
static_assert(sizeof(Engine) % 4 == 0 && sizeof(Stats) % 4 == 0, "checkpoints are copied by words");

struct Move {
    int orient, x, hold;
    bool none;
    uint64_t key1, key2;               // tracing flavour: the final argmax's two largest keys
};

struct LevelAcc {
    uint64_t thr;                      // list[k-1], the key a candidate must beat
    uint64_t list;                     // top-K list (STAGE_TOPK)
    uint64_t best;                     // argmax of leaf keys and fallbacks (STAGE_LEAF)
    uint64_t best2;                    // the second-largest leaf key (tracing flavour only)
    uint32_t lo, hi;                   // TOPK: bit k = parent k has a legal child; LEAF: bit = list legal
};

// keep the two largest keys (keys are unique per move, 0 = none)
__device__ __forceinline__ void top2_insert(uint64_t& b1, uint64_t& b2, uint64_t k) {
    if (k > b1) {
        b2 = b1;
        b1 = k;
    } else if (k > b2) {
        b2 = k;
    }
}

// the two largest keys over the warp, in every lane (each step merges disjoint lane sets)
__device__ __forceinline__ void warp_top2(uint64_t& b1, uint64_t& b2) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        int const src = int((threadIdx.x + o) & 31u);
        uint64_t const u1 = shfl64(b1, src), u2 = shfl64(b2, src);
        uint64_t const lo = b1 < u1 ? b1 : u1, hi2 = b2 > u2 ? b2 : u2;
        b1 = b1 > u1 ? b1 : u1;
        b2 = lo > hi2 ? lo : hi2;
    }
}

__device__ __forceinline__ uint64_t candidate_key(bool leaf, float v, uint32_t info, uint32_t i) {
    uint32_t const k = (info >> 8) & 31u, child = (info >> 21) & 1u;
    uint32_t const pos = (k * 2u + child) * MP + i;                        // beam.hpp:296,360,423
    uint32_t const low = leaf ? uint32_t(ORDER_SPAN) - pos : 0xFFFFFFFFu - pos;   // beam.hpp:217-219
    return (uint64_t(ordered_bits(v)) << 32) | uint64_t(low);
}

struct Luts {
    PlaceFast const (*fast)[MP];
    uint32_t const (*move)[MP];
};

// Full path for one queued candidate (segment << 8 | placement): its key, or 0 if illegal.
// A legal candidate's key is never 0 (its low word is a positive position).
__device__ __noinline__ uint64_t full_key(WarpShared* ws, Luts lut, bool leaf, uint32_t entry) {
    uint32_t const seg = entry >> 8, i = entry & 0xFFu;
    uint32_t const info = ws->seg_info[seg];
    uint32_t const* rec = ws->rec[info & 63u];
    uint32_t const mv = lut.move[(info >> 16) & 7u][i];
    Applied const a = apply_ints(rec + R_BOARD, mv & 0xFFFFu, int((mv >> 16) & 0xFu), nullptr);
    if (!a.legal) return 0;
    float const v = value_full(rec[R_CLEARS] + clear_bump(a.cleared), a.bi, (info >> 20) & 1u, SmemW{ws->wfull});
    return candidate_key(leaf, v, info, i);
}

// The widened network's full path, first half: is the queued candidate legal,
// and its inputs (all zero when it is not).
__device__ __noinline__ bool full_inputs_wide(WarpShared* ws, Luts lut, uint32_t entry, WideIn& in) {
    uint32_t const seg = entry >> 8, i = entry & 0xFFu;
    uint32_t const info = ws->seg_info[seg];
    uint32_t const* rec = ws->rec[info & 63u];
    uint32_t const mv = lut.move[(info >> 16) & 7u][i];
    Applied const a = apply_ints(rec + R_BOARD, mv & 0xFFFFu, int((mv >> 16) & 0xFu), nullptr);
    if (!a.legal) return false;
    wide_inputs(rec[R_CLEARS] + clear_bump(a.cleared), a.bi, (info >> 20) & 1u, in.v);
    return true;
}

// One level: every candidate of the segment table, on the fast path or queued
// for the full path (evaluated in compacted 32-lane batches). leaf: fold into
// the argmax key and per-list legality; otherwise into the top-kl list and
// per-parent legality. ws is the game's area, own the warp's own (its queue of deferred
// candidates and its key buffer; the same area except in team kernels).
// TEAM > 1: this warp takes every TEAM-th 32-candidate round, starting at candidate `first`.
//
// The top-kl list (lane i = i-th largest, 0 = empty; thr = list[kl-1]): keys are unique per level
// (the low word encodes the slot), so the kept set equals beam.hpp:244-265's "max score, lowest
// slot on ties" whatever the order keys arrive in. The single-warp kernels insert each key above
// thr at once (topk_fold). The team kernels keep the list lazily: keys above thr go to the
// warp's key buffer, and when a round's keys would overflow it (or the level ends) the buffer is
// sorted across the lanes and merged into the list, which raises thr; a key at or below a stale
// thr is below the final list[kl-1] too. The lazy merge shortens a warp's critical path (15 %
// per move for a warp alone on its scheduler) but executes more instructions, which costs 3-5 %
// at 16 warps per SM, where the single-warp kernels run.
template <int NET, bool KEYS, int TEAM = 1>
__device__ __forceinline__ LevelAcc level_pass(WarpShared& ws, WarpShared& own, Luts lut, FastW const& fw, float* hb,
                                               bool leaf, uint32_t total, int kl, int lane, uint32_t& evals,
                                               uint32_t first = 0) {
    constexpr bool WIDE = NET != 0;
    constexpr int HW = WIDE ? NET : 64;     // the widened network's width (unused for v11)
    uint32_t* const dq = own.defer;
    uint64_t* const kb = own.kbuf;
    constexpr bool TEAMED = TEAM > 1;
    constexpr bool LAZY = TEAMED;
    LevelAcc acc{0, 0, 0, 0, 0, 0};
    auto consume = [&](uint64_t key, uint32_t seg, uint32_t info) {
        if (key) {
            ++evals;
            uint32_t const bit = leaf ? seg : (info >> 8) & 31u;
            if (bit < 32) acc.lo |= 1u << bit;
            else acc.hi |= 1u << (bit - 32);
        }
    };
    // Each iteration is one round of 32 fast-path candidates (one per lane) or, once 32 are
    // queued (or the level is done), one batch of up to 32 deferred candidates through the full
    // path; either way its keys are folded at one place. Keys are unique within a level, so the
    // fold order does not change the kept set. One drain site and one fold site keep the loop's
    // code small (the kernel is bound by instruction fetch as much as by issue). Two candidates
    // per lane in straight-line code measured slower (681 ms vs 486 ms per full generation).
    uint32_t queued = 0;          // < 32 at the start of every fast round: the queue holds 64
    uint32_t kcnt = 0;            // keys in the key buffer (non-leaf levels)
    int seg = 0;
    uint32_t c0 = TEAMED ? first : 0u;
    for (;;) {
        bool const more = c0 < total;
        // the level's candidates are done; a non-leaf level takes one more turn to merge its buffer
        bool const fin = !more && queued == 0;
        if (fin && (leaf || !LAZY || kcnt == 0)) break;
        uint64_t key = 0;
        if (fin) {
        } else if (queued >= uint32_t(WARP) || !more) {
            // ---- a batch of deferred candidates through the full reference path
            uint32_t const n = queued < uint32_t(WARP) ? queued : uint32_t(WARP);
            __syncwarp();
            if constexpr (WIDE) {
                // the inputs per lane, then the network on all lanes together
                WideIn in{};
                uint32_t entry = 0;
                bool legal = false;
                if (uint32_t(lane) < n) {
                    entry = dq[lane];
                    legal = full_inputs_wide(&ws, lut, entry, in);
                    if (!legal) in = WideIn{};
                }
                __syncwarp();
                float const v = wide_value<HW>(in, ws.wglobal, hb, lane);
                if (legal) {
                    uint32_t const info = ws.seg_info[entry >> 8];
                    key = candidate_key(leaf, v, info, entry & 0xFFu);
                    consume(key, entry >> 8, info);
                }
            } else if (uint32_t(lane) < n) {
                uint32_t const entry = dq[lane];
                key = full_key(&ws, lut, leaf, entry);
                consume(key, entry >> 8, ws.seg_info[entry >> 8]);
            }
            uint32_t const rem = queued - n;
            uint32_t t = 0;
            __syncwarp();
            if (uint32_t(lane) < rem) t = dq[n + lane];
            __syncwarp();
            if (uint32_t(lane) < rem) dq[lane] = t;
            __syncwarp();
            queued = rem;
        } else {
            // ---- a round of fast-path candidates
            uint32_t const c = c0 + uint32_t(lane);
            bool const valid = c < total;
            uint32_t const cc = valid ? c : total - 1u;          // out of range: the last candidate, discarded
            while (ws.seg_off[seg + 1] <= cc) ++seg;
            uint32_t const sg = uint32_t(seg);
            uint32_t const info = ws.seg_info[seg];
            uint32_t const idx = cc - ws.seg_off[seg];
            float v;
            int st;
            if constexpr (WIDE)
                st = fast_candidate_wide<HW>(ws.rec[info & 63u], lut.fast[(info >> 16) & 7u][idx], (info >> 20) & 1u,
                                             ws.wglobal, hb, lane, v);
            else
                st = fast_candidate(ws.rec[info & 63u], lut.fast[(info >> 16) & 7u][idx], (info >> 20) & 1u, fw, v);
            bool const def = valid && st != FAST_OK;
            if (valid && st == FAST_OK) {
                key = candidate_key(leaf, v, info, idx);
                consume(key, sg, info);
            }
            uint32_t const dm = __ballot_sync(FULL_MASK, def);
            if (def) dq[queued + __popc(dm & ((1u << lane) - 1u))] = (sg << 8) | idx;
            queued += __popc(dm);
            c0 += uint32_t(TEAM * WARP);
        }
        if (leaf) {
            if (KEYS) top2_insert(acc.best, acc.best2, key);
            else acc.best = key > acc.best ? key : acc.best;
        } else if (!LAZY) {
            topk_fold(acc.list, acc.thr, key, kl, lane);
        } else {
            uint32_t m = __ballot_sync(FULL_MASK, key > acc.thr);
            uint32_t n = __popc(m);
            if (fin || kcnt + n > uint32_t(WARP)) {          // merge the buffer into the list
                __syncwarp();
                uint64_t const b = warp_sort_desc(uint32_t(lane) < kcnt ? kb[lane] : 0ull, lane);
                acc.list = merge_topk(acc.list, b, kl, lane);
                acc.thr = shfl64(acc.list, kl - 1);
                kcnt = 0;
                m = __ballot_sync(FULL_MASK, key > acc.thr);
                n = __popc(m);
                __syncwarp();
            }
            if (key > acc.thr) kb[kcnt + __popc(m & ((1u << lane) - 1u))] = key;
            kcnt += n;
        }
    }
    return acc;
}

// Segment table of one level: segment j = (parent rank j/2, child list j%2),
// spanning the child piece's placement count. Returns the candidate total.
__device__ __forceinline__ uint32_t build_segments(WarpShared& ws, uint32_t const* slot_piece, int tree, int level,
                                                   uint32_t fnode, int kept, int lane) {
    uint32_t base = 0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        int const j = lane + 32 * half;
        int const k = j >> 1;
        uint32_t const pnode = __shfl_sync(FULL_MASK, fnode, k & 31);
        uint32_t const cnode = (2u * pnode + uint32_t(j & 1)) & 15u;
        uint32_t const nd = c_tables.node[tree][level][cnode];
        uint32_t const piece = slot_piece[nd & 0xFu];
        uint32_t const held_slot = (nd >> 4) & 0xFu;
        uint32_t const held_i = held_slot != HELD_NONE && slot_piece[held_slot] == 0u;
        uint32_t const cnt = k < kept ? c_tables.nplace[piece] : 0u;
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t const n = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= o) incl += n;
        }
        ws.seg_off[j] = base + incl - cnt;
        ws.seg_info[j] = uint32_t(k & 31) | (uint32_t(k & 31) << 8) | (piece << 16) | (held_i << 20) |
                         (uint32_t(j & 1) << 21);
        base += __shfl_sync(FULL_MASK, incl, 31);
    }
    if (lane == 0) ws.seg_off[64] = base;
    __syncwarp();
    return base;
}

// lane j builds kept node j (when active): parent record `prec`, placement (piece, i); with
// root, the active lane builds record 32 from the committed board (no placement, no clears)
template <bool WIDE>
__device__ __noinline__ void materialize(WarpShared* ws, Luts lut, bool active, uint32_t prec, uint32_t piece,
                                         uint32_t i, int lane, bool root = false) {
    uint32_t nb[W];
    uint32_t ncl = 0;
    if (active && root) {
        load_board(ws->eng.board, nb);
    } else if (active) {
        uint32_t const* pr = ws->rec[prec];
        uint32_t b[W];
        load_board(pr + R_BOARD, b);
        uint32_t const mv = lut.move[piece][i];
        int cl = 0;
        apply_full(b, mv & 0xFFFFu, int((mv >> 16) & 0xFu), nb, cl);
        ncl = pr[R_CLEARS] + clear_bump(cl);
    }
    __syncwarp();
    if (active) build_record<SmemW, !WIDE>(nb, ncl, SmemW{ws->wfull}, ws->rec[root ? 32 : lane]);
    __syncwarp();
}

// the committed board's record (record 32): one lane builds it through materialize's body, so the
// kernel holds one copy of the record builder (a second inlined copy measured 5 % slower on the
// headline generation: the kernel is bound by instruction fetch as much as by issue)
template <bool WIDE>
__device__ __forceinline__ void root_record(WarpShared* ws, Luts lut, int lane) {
    materialize<WIDE>(ws, lut, lane == 0, 0u, 0u, 0u, lane, true);
}

// search_move_beam (beam.hpp:484-570) for the warp's committed game.
// TEAM > 1: ws is the team's game (the leader's area, the partners' follow it). The leader runs
// the search and posts each stage; a partner stays in here for the whole game, runs the stages it
// is posted (its share of each candidate pass) and returns when the leader posts TEAM_GAME_END.
template <int NET, bool KEYS, int TEAM = 1>
__device__ __forceinline__ Move search_move(WarpShared& ws, Luts lut, FastW const& fw, float* hb, int lane, uint32_t& evals,
                                            uint32_t* status) {
    constexpr bool WIDE = NET != 0;
    constexpr bool TEAMED = TEAM > 1;
    static_assert(!TEAMED || (!WIDE && !KEYS), "team kernels run the v11 model without key tracing");
    int const rank = TEAMED ? int((threadIdx.x >> 5) & uint32_t(TEAM - 1)) : 0;
    bool const partner = rank != 0;
    WarpShared* const pr = &ws;
    Move mv{0, 0, 0, true, 0, 0};
    if (!partner && ws.eng.over) return mv;
    uint32_t slot_piece[NSLOTS];                                  // beam.hpp:226-237
    int tree = 0;
    uint32_t r0 = 0, r1 = 0, p0 = 0, p1 = 0;
    if (!partner) {
        slot_piece[0] = ws.eng.held;
        slot_piece[1] = ws.eng.queue[0];
#pragma unroll
        for (int i = 0; i < DEPTH; ++i) slot_piece[2 + i] = ws.eng.queue[1 + i];
        tree = ws.eng.held == NO_PIECE ? 1 : 0;
        r0 = c_tables.node[tree][0][0];
        r1 = c_tables.node[tree][0][1];
        p0 = slot_piece[r0 & 0xFu];
        p1 = slot_piece[r1 & 0xFu];
    }

    int kept = 1;                              // frontier size feeding the next stage
    uint32_t fscore = 0, fnode = 0, frank = uint32_t(lane), root_slot = 0;
    uint64_t best = 0;                         // leaf-order (score | order) maximum, fallbacks included
    uint64_t best2 = 0;                        // the second-largest such key (tracing flavour)
#pragma unroll 1
    for (int stage = 0;; ++stage) {
        // ---- segments of this stage
        uint32_t total;
        if (partner) {                         // the stage the leader posts, or the end of the game
            if (!team_sync(pr, rank, status, lane)) return mv;
            uint32_t const cmd = ws.team_cmd;
            if (cmd == TEAM_GAME_END) return mv;
            stage = int(cmd);
            total = ws.team_total;
        } else if (stage == DEPTH) {
            break;
        } else if (stage == 0) {               // two root groups over the committed board (beam.hpp:283-301)
            root_record<WIDE>(&ws, lut, lane);
            if (lane < 2) {
                uint32_t const nd = lane ? r1 : r0;
                uint32_t const held_slot = (nd >> 4) & 0xFu;
                uint32_t const held_i = held_slot != HELD_NONE && slot_piece[held_slot] == 0u;
                ws.seg_info[lane] = 32u | ((lane ? p1 : p0) << 16) | (held_i << 20) | (uint32_t(lane) << 21);
            }
            total = c_tables.nplace[p0] + c_tables.nplace[p1];
            if (lane == 0) {
                ws.seg_off[0] = 0;
                ws.seg_off[1] = c_tables.nplace[p0];
                ws.seg_off[2] = total;
                ws.seg_off[3] = total;
            }
            __syncwarp();
        } else {
            total = build_segments(ws, slot_piece, tree, stage, fnode, kept, lane);
        }
        if (TEAMED && !partner) {                // post the stage
            if (lane == 0) {
                ws.team_cmd = uint32_t(stage);
                ws.team_total = total;
            }
            if (!team_sync(pr, 0, status, lane)) return mv;
        }
        bool const leaf = stage == DEPTH - 1;
        int const kl = stage == 0 ? K0 : (stage == 1 ? K1 : K2);
        // ---- every candidate of the stage
        // team kernels reload the fast-path weights for each pass (from L1), so that they hold no
        // registers across the team barriers
        FastW fwl;
        if (TEAMED) load_fast_weights(GlobalW{ws.wglobal}, fwl);
        LevelAcc a = level_pass<NET, KEYS, TEAM>(ws, pr[rank], lut, TEAMED ? fwl : fw, hb, leaf, total, kl, lane, evals,
                                                 uint32_t(rank * WARP));
        if (TEAMED) {
            // a partner's results go through its own record area, which it never uses otherwise
            if (partner) {
                uint32_t* const x = pr[rank].rec[0];
                reinterpret_cast<uint64_t*>(x)[lane] = leaf ? a.best : a.list;
                uint32_t const lo = __reduce_or_sync(FULL_MASK, a.lo), hi = __reduce_or_sync(FULL_MASK, a.hi);
                if (lane == 0) {
                    x[X_LO] = lo;
                    x[X_HI] = hi;
                }
                if (!team_sync(pr, rank, status, lane)) return mv;
                continue;
            }
            if (!team_sync(pr, 0, status, lane)) return mv;
#pragma unroll 1
            for (int m = 1; m < TEAM; ++m) {
                uint32_t const* const x = pr[m].rec[0];
                uint64_t const b = reinterpret_cast<uint64_t const*>(x)[lane];
                if (leaf) a.best = b > a.best ? b : a.best;
                else a.list = merge_topk(a.list, b, kl, lane);
                a.lo |= x[X_LO];
                a.hi |= x[X_HI];
            }
        }
        if (stage == 0) {
            // ---- seed the frontier with the selected roots (beam.hpp:307-329): lane k = rank k
            kept = __popc(__ballot_sync(FULL_MASK, a.list != 0));
            if (kept == 0) return mv;                             // no legal root: game over
            root_slot = 0xFFFFFFFFu - uint32_t(a.list);
            fscore = uint32_t(a.list >> 32);
            uint32_t const g = lane < kept ? root_slot / MP : 0u;
            fnode = g;
            materialize<WIDE>(&ws, lut, lane < kept, 32u, g ? p1 : p0, root_slot % MP, lane);
        } else if (!leaf) {
            uint32_t const has_child = __reduce_or_sync(FULL_MASK, a.lo);
            // kept nodes with no legal continuation become leaves at this depth (beam.hpp:549-551)
            if (lane < kept && !((has_child >> lane) & 1u)) {
                uint64_t const fk = (uint64_t(fscore) << 32) | uint64_t(ORDER_SPAN - (LEAF_ORDERS + frank));
                if (KEYS) top2_insert(best, best2, fk);
                else best = fk > best ? fk : best;
            }
            int const next = __popc(__ballot_sync(FULL_MASK, a.list != 0));
            // advance the frontier (beam.hpp:379-403): lane j builds kept node j
            uint32_t const sslot = 0xFFFFFFFFu - uint32_t(a.list);
            uint32_t const pk = lane < next ? sslot / (2 * MP) : 0u;
            uint32_t const child = (sslot / MP) & 1u;
            uint32_t const par_node = __shfl_sync(FULL_MASK, fnode, int(pk));
            uint32_t const par_rank = __shfl_sync(FULL_MASK, frank, int(pk));
            uint32_t const cnode = (2u * par_node + child) & 15u;
            uint32_t const piece = slot_piece[c_tables.node[tree][stage][cnode] & 0xFu];
            materialize<WIDE>(&ws, lut, lane < next, pk, piece, sslot % MP, lane);
            fscore = uint32_t(a.list >> 32);
            fnode = lane < next ? cnode : 0u;
            frank = par_rank;
            kept = next;
        } else {
            // ---- leaf stage (beam.hpp:407-443): a list whose piece never fit scores the frontier board
            uint32_t const legal_lo = __reduce_or_sync(FULL_MASK, a.lo);
            uint32_t const legal_hi = __reduce_or_sync(FULL_MASK, a.hi);
            if (KEYS) {
                top2_insert(best, best2, a.best);
                top2_insert(best, best2, a.best2);
            } else {
                best = a.best > best ? a.best : best;
            }
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                int const j = lane + 32 * half;
                int const k = j >> 1;
                uint32_t const sc = __shfl_sync(FULL_MASK, fscore, k & 31);
                bool const legal = ((half ? legal_hi : legal_lo) >> lane) & 1u;
                if (k < kept && !legal) {
                    uint64_t const key = (uint64_t(sc) << 32) | uint64_t(ORDER_SPAN - uint32_t(j) * MP);
                    if (KEYS) top2_insert(best, best2, key);
                    else best = key > best ? key : best;
                }
            }
        }
    }
    if (KEYS) {
        warp_top2(best, best2);
        mv.key1 = best;
        mv.key2 = best2;
    } else {
        best = warp_max64(best);
    }
    if (best == 0) {                                              // unreachable with >= 1 root
        if (lane == 0) atomicOr(status, 1u);
        return mv;
    }
    // ---- decode the winning key back to its root move (beam.hpp:450-470)
    uint32_t const order = ORDER_SPAN - uint32_t(best);
    uint32_t const leaf_rank = __shfl_sync(FULL_MASK, frank, int((order / (2 * MP)) & 31u));
    uint32_t const root_rank = order >= uint32_t(LEAF_ORDERS) ? order - LEAF_ORDERS : leaf_rank;
    uint32_t const rs = __shfl_sync(FULL_MASK, root_slot, int(root_rank & 31u));
    uint32_t const g = rs / MP;
    uint32_t const pa = lut.move[g ? p1 : p0][rs % MP];
    mv.orient = int((pa >> 20) & 3u);
    mv.x = int((pa >> 24) & 0xFu) - 2;
    mv.hold = int((c_tables.node[tree][0][g] >> 8) & 1u);
    mv.none = ordered_bits_inv(uint32_t(best >> 32)) == -__int_as_float(0x7f800000);   // search.hpp:41
    return mv;
}

// Checkpoint the warp's game for the paired kernel: engine and stats, the sim (parked in the warp's
// team_sim word), its moves (= pieces placed: the game goes on, so no move failed) and evaluation
// count (the provisional result the warp wrote). false when the array is full.
__device__ __noinline__ bool save_checkpoint(WarpShared* ws, uint32_t* scratch, Checkpoint* ckpt, uint32_t cap,
                                             uint32_t const* evals, int lane) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(&scratch[kCkptCountWord], 1u);
    idx = __shfl_sync(FULL_MASK, idx, 0);
    if (idx >= cap) return false;
    Checkpoint* const c = ckpt + idx;
    uint32_t const* const e = reinterpret_cast<uint32_t const*>(&ws->eng);
    uint32_t const* const t = reinterpret_cast<uint32_t const*>(&ws->st);
    for (int i = lane; i < int(sizeof(Engine) / 4); i += WARP) reinterpret_cast<uint32_t*>(&c->eng)[i] = e[i];
    for (int i = lane; i < int(sizeof(Stats) / 4); i += WARP) reinterpret_cast<uint32_t*>(&c->st)[i] = t[i];
    __syncwarp();
    if (lane == 0) {
        uint32_t const sim = ws->team_sim;
        c->eng.over = 0;                                // (ws->eng.over holds the hand-off marker)
        c->sim = sim;
        c->moves = ws->st.pieces;                       // every committed move placed one piece
        c->evals = evals ? evals[sim] : 0u;             // the provisional result the warp just wrote
    }
    return true;
}

// A team kernel's resume: the leader warp takes the checkpointed game's state.
__device__ __noinline__ void load_checkpoint(WarpShared* ws, Checkpoint const* c, int lane) {
    uint32_t* const e = reinterpret_cast<uint32_t*>(&ws->eng);
    uint32_t* const t = reinterpret_cast<uint32_t*>(&ws->st);
    for (int i = lane; i < int(sizeof(Engine) / 4); i += WARP) e[i] = reinterpret_cast<uint32_t const*>(&c->eng)[i];
    for (int i = lane; i < int(sizeof(Stats) / 4); i += WARP) t[i] = reinterpret_cast<uint32_t const*>(&c->st)[i];
    __syncwarp();
}

// NET: 0 = the v11 model; H = the widened 10 -> H -> H -> 1 network (64: 4,929 weights per
// model, 32: 1,441) instead of v11.
// BUDGET: the flavour that checks the launch's time budget after every move (a separate
// instantiation: the check's registers would otherwise cost the ordinary kernels spills).
// KEYS: the tracing flavour that also records each move's two largest final keys (p.keys).
// TEAM: warps per game; TEAM > 1 (v11 only, no budget, no key tracing): the team's first warp
// takes the tickets, commits the moves and writes the results, the others run their share of
// every candidate pass (search_move's team mode); results are the single-warp kernel's, bit for
// bit. With p.resume it plays the games a HANDOFF launch checkpointed.
// HANDOFF: the launch's tail goes to a team kernel. A warp that finds no sim left counts itself
// done; when at most p.handoff_at warps still play, it raises the hand-off flag, and every playing
// warp then checkpoints its game at its next move boundary (checked every 4th move) and ends; the
// team kernel, launched next on the same stream, finishes those games.
template <int WARPS, int MINB, int NET = 0, bool BUDGET = false, bool KEYS = false, int TEAM = 1,
          bool HANDOFF = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) eval_kernel(Params p) {
    constexpr bool WIDE = NET != 0;
    constexpr int HW = WIDE ? NET : 64;
    constexpr bool TEAMED = TEAM > 1;
    static_assert(TEAM == 1 || TEAM == 2 || TEAM == 4 || TEAM == 8, "teams of 1, 2, 4 or 8 warps");
    static_assert(!TEAMED || (!WIDE && !BUDGET && !KEYS && WARPS % TEAM == 0), "team kernels: v11, whole teams");
    static_assert(!HANDOFF || (!WIDE && !BUDGET && !KEYS && !TEAMED), "hand-off: the single-warp v11 kernel");
    extern __shared__ __align__(16) unsigned char dyn_smem[];    // WARPS x WarpShared
    __shared__ LutTables s_lut;
    for (int t = int(threadIdx.x); t < NPIECE * MP; t += WARPS * 32) {
        s_lut.fast[t / MP][t % MP] = g_lut.fast[t / MP][t % MP];
        s_lut.move[t / MP][t % MP] = g_lut.move[t / MP][t % MP];
    }
    int const lane = int(threadIdx.x & 31u);
    int const rank = TEAMED ? int((threadIdx.x >> 5) & uint32_t(TEAM - 1)) : 0;
    bool const partner = rank != 0;
    // TEAM > 1: pr[0] is the team's game (the leader's area), pr[r] warp r's area
    WarpShared* const pr = reinterpret_cast<WarpShared*>(dyn_smem) + ((threadIdx.x >> 5) & ~uint32_t(TEAM - 1));
    WarpShared& ws = pr[0];
    if (TEAMED && lane == 0) {
        if (!partner) team_bar_init(pr, uint32_t(TEAM));
        pr[rank].team_broken = 0;
    }
    if (HANDOFF && lane == 0) ws.eng.over = 0;                 // (read after the game loop)
    __syncthreads();
    if (TEAMED && partner && (p.test_flags & 1u)) return;      // (no later block barrier)
    Luts const lut{s_lut.fast, s_lut.move};
    // the widened network's per-warp hidden-unit buffers follow the WARPS warp blocks
    float* const hb = WIDE ? reinterpret_cast<float*>(dyn_smem + WARPS * sizeof(WarpShared)) +
                                 (threadIdx.x >> 5) * kWideHbFloats<HW>
                           : nullptr;
    // time budget, measured from this warp's start (the persistent grid starts every warp at launch);
    // kept in shared memory so it costs no register in the move loop
    if (BUDGET && lane == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ws.t_start));
    for (;;) {
        // a 64-bit ticket: every resident warp draws one past the last sim, which a 32-bit
        // counter could wrap near 2^32 sims; kNoSim (no sim index is that large) ends the warp
        uint32_t sim = 0, ck = 0;
        if (!partner && lane == 0) {
            sim = kNoSim;
            if (TEAMED && p.resume) {
                // the checkpointed games, spread over the blocks
                uint32_t n = *reinterpret_cast<volatile uint32_t*>(&p.scratch[kCkptCountWord]);
                n = n < p.ckpt_cap ? n : p.ckpt_cap;
                if ((threadIdx.x >> 5) / uint32_t(TEAM) < (n + gridDim.x - 1) / gridDim.x) {
                    ck = atomicAdd(&p.scratch[kCkptTicketWord], 1u);
                    if (ck < n) sim = p.ckpt[ck].sim;
                }
            } else if (!p.warps_active || (threadIdx.x >> 5) < p.warps_active) {
                // (a warp beyond the block's playing warps takes no ticket: the batch is spread over the SMs)
                unsigned long long const t = atomicAdd(reinterpret_cast<unsigned long long*>(p.scratch), 1ull);
                if (t < p.total_sims) sim = uint32_t(t);
            }
            if (HANDOFF && sim == kNoSim) {
                uint32_t const total = gridDim.x * (p.warps_active ? p.warps_active : uint32_t(WARPS));
                uint32_t const done = atomicAdd(&p.scratch[kDoneWord], 1u) + 1u;
                if (total - done <= p.handoff_at) atomicExch(&p.scratch[kHandoffWord], 1u);
            }
        }
        if (TEAMED) {                                                // the leader hands the sim to its partners
            if (!partner && lane == 0) ws.team_sim = sim;
            if (!team_sync(pr, rank, &p.scratch[kStatusWord], lane)) break;
            sim = __shfl_sync(FULL_MASK, ws.team_sim, 0);
        } else {
            sim = __shfl_sync(FULL_MASK, sim, 0);
        }
        if (sim == kNoSim) break;
        uint32_t const mdl = sim / p.num_games, g = sim % p.num_games;
        uint32_t const island = mdl / p.models_per_island;
        uint64_t const seed = p.seeds[size_t(island) * p.num_games + g];
        float const* wsrc = p.weights + size_t(mdl) * (WIDE ? WideNet<HW>::STRIDE : NPARAMS);
        bool const resumed = TEAMED && p.resume;
        if (p.timing && lane == 0 && !resumed) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            p.timing[2 * size_t(sim)] = t;
        }
        FastW fw;
        uint32_t evals = 0, moves = 0;
        if (!WIDE) load_fast_weights(GlobalW{wsrc}, fw);
        if (!partner) {
            if (!WIDE)
                for (int i = lane; i < NPARAMS; i += WARP) ws.wfull[i] = __ldg(wsrc + i);
            if (lane == 0) {
                ws.wglobal = wsrc;
                if (HANDOFF) ws.team_sim = sim;                    // (read by the hand-off's checkpoint)
            }
            if (resumed) {
                Checkpoint const* const c = p.ckpt + __shfl_sync(FULL_MASK, ck, 0);
                load_checkpoint(&ws, c, lane);
                moves = c->moves;
                if (lane == 0) evals = c->evals;
            } else if (lane == 0) {
                engine_reset(ws.eng, seed);
                ws.st = Stats{};
            }
        }
        __syncwarp();
        // team kernels: a partner's one search_move call serves the whole game (it returns when the
        // leader ends the game), so both roles run the same copy of the search code
        while (partner || (moves < p.max_moves && !ws.eng.over)) {   // model_eval_host.cpp:39-50
            Move const mv = search_move<NET, KEYS, TEAM>(ws, lut, fw, hb, lane, evals, &p.scratch[kStatusWord]);
            if (partner) break;
            if (TEAMED && ws.team_broken) break;
            if (KEYS && lane == 0 && p.keys) {
                p.keys[(size_t(sim) * p.max_moves + moves) * 2] = mv.key1;
                p.keys[(size_t(sim) * p.max_moves + moves) * 2 + 1] = mv.key2;
            }
            if (mv.none) break;
            if (lane == 0) {
                if (p.trace) {
                    uint8_t* t = p.trace + (size_t(sim) * p.max_moves + moves) * 3;
                    t[0] = uint8_t(mv.hold);
                    t[1] = uint8_t(mv.orient);
                    t[2] = uint8_t(mv.x + 2);
                }
                if (mv.hold) engine_hold(ws.eng);
                BoardInts bi;
                int const cl = engine_place(ws.eng, mv.orient, mv.x, bi);
                if (cl >= 0) stats_advance(ws.st, bi, uint32_t(cl));
                else ws.eng.over = 2;                                // DIED: stop without a stats update
            }
            ++moves;
            __syncwarp();
            if (ws.eng.over == 2) break;
            if (HANDOFF && (moves & 3u) == 0 && moves < p.max_moves && !ws.eng.over) {
                uint32_t f = 0;
                if (lane == 0) f = *reinterpret_cast<volatile uint32_t*>(&p.scratch[kHandoffWord]);
                if (__shfl_sync(FULL_MASK, f, 0)) {
                    if (lane == 0) ws.eng.over = 4;                  // handed over after the game loop
                    __syncwarp();
                    break;
                }
            }
            if (BUDGET) {                                          // over = 3: out of time, stop here
                if (lane == 0) {
                    unsigned long long now;
                    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
                    if (now - ws.t_start > p.budget_ns) {
                        atomicOr(&p.scratch[kStatusWord], 2u);
                        ws.eng.over = 3;
                    }
                }
                __syncwarp();
                if (ws.eng.over == 3) break;
            }
        }
        if (TEAMED) {                           // the leader ends the partners' game and takes their counts
            if (pr[rank].team_broken) break;
            if (!partner) {
                if (lane == 0) ws.team_cmd = TEAM_GAME_END;
                if (!team_sync(pr, 0, &p.scratch[kStatusWord], lane)) break;
            } else {
                uint32_t const own = __reduce_add_sync(FULL_MASK, evals);
                if (lane == 0) pr[rank].rec[0][X_EVALS] = own;
            }
            if (!team_sync(pr, rank, &p.scratch[kStatusWord], lane)) break;
            if (partner) continue;
        }
        evals = __reduce_add_sync(FULL_MASK, evals);
        if (TEAMED)
#pragma unroll 1
            for (int m = 1; m < TEAM; ++m) evals += pr[m].rec[0][X_EVALS];
        if (lane == 0) {
            p.score[sim] = final_score(ws.st);
            if (p.pieces) p.pieces[sim] = ws.st.pieces;
            if (p.lines) p.lines[sim] = ws.st.lines;
            if (p.evals) p.evals[sim] = evals;
            if (p.n_moves) p.n_moves[sim] = moves;
            if (p.board_out)
                for (int x = 0; x < W; ++x) p.board_out[size_t(sim) * W + x] = ws.eng.board[x];
            if (p.timing) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                p.timing[2 * size_t(sim) + 1] = t;
            }
        }
        __syncwarp();
        if (BUDGET && ws.eng.over == 3) break;                   // out of time: take no further sim
    }
    // The paired kernel finishes a handed-over game (over = 4; the game's results written above are
    // provisional: the paired kernel overwrites them). At most handoff_at <= ckpt_cap games are
    // still playing when the flag rises, so a full array is an error.
    if (HANDOFF && ws.eng.over == 4) {
        __syncwarp();
        if (!save_checkpoint(&ws, p.scratch, p.ckpt, p.ckpt_cap, p.evals, lane) && lane == 0)
            atomicOr(&p.scratch[kStatusWord], 8u);
    }
}

// Device self-test of the candidate core (tests only): one thread per
// candidate, fast path and full path on caller-built records. cand[t] =
// piece | placement << 8 | held-is-I << 16 | record index << 17.
__global__ void core_selftest_kernel(uint32_t const* recs, uint32_t const* cand, uint32_t n, float const* w,
                                     float* fast_v, int* fast_st, float* full_v, int* full_legal, float* dbg) {
    uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint32_t const c = cand[t];
    uint32_t const piece = c & 0xFFu, i = (c >> 8) & 0xFFu, held = (c >> 16) & 1u;
    uint32_t const* rec = recs + size_t(c >> 17) * REC_WORDS;
    FastW fw;
    load_fast_weights(GlobalW{w}, fw);
    float v = 0.0f;
    // the kernel's own arithmetic mode, then (diagnostics) every MLP mode: scalar, packed
    // intrinsics, packed PTX
    fast_st[t] = fast_candidate(rec, g_lut.fast[piece][i], held, fw, v, dbg ? dbg + size_t(t) * 32 : nullptr);
    if (dbg) {
        float v2 = 0.0f, v3 = 0.0f, v4 = 0.0f, v5 = 0.0f;
        fast_candidate<MLP_PTX_X2>(rec, g_lut.fast[piece][i], held, fw, v2, nullptr);
        fast_candidate<MLP_X2>(rec, g_lut.fast[piece][i], held, fw, v3, nullptr);
        fast_candidate<MLP_SCALAR>(rec, g_lut.fast[piece][i], held, fw, v4, nullptr);
        fast_candidate<MLP_X2MUL>(rec, g_lut.fast[piece][i], held, fw, v5, nullptr);
        dbg[size_t(t) * 32 + 28] = v5;
        dbg[size_t(t) * 32 + 29] = v4;
        dbg[size_t(t) * 32 + 30] = v3;
        dbg[size_t(t) * 32 + 31] = v2;
    }
    fast_v[t] = v;
    uint32_t const mv = g_lut.move[piece][i];
    uint32_t b[W], nb[W];
    for (int x = 0; x < W; ++x) b[x] = rec[R_BOARD + x];
    int cl = 0;
    full_legal[t] = apply_full(b, mv & 0xFFFFu, int((mv >> 16) & 0xFu), nb, cl);
    full_v[t] = full_legal[t] ? value_full(rec[R_CLEARS] + clear_bump(cl), board_ints(nb), held, GlobalW{w}) : 0.0f;
}

// widened models -> their device layout (WideNet<H>::STRIDE floats per model: layers
// 1 and 2 transposed, SKIP = 1 when zero terms may be left out). One block per model.
template <int H>
__global__ void repack_wide_kernel(float const* __restrict__ src, uint32_t models, float* __restrict__ dst) {
    using D = WideNet<H>;
    uint32_t const m = blockIdx.x;
    if (m >= models) return;
    float const* s = src + size_t(m) * D::N;
    float* d = dst + size_t(m) * D::STRIDE;
    int ok = 1;
    for (int j = int(threadIdx.x); j < D::N; j += int(blockDim.x)) {
        float const x = s[j];
        ok &= isfinite(x) && !(D::is_bias(j) && x == 0.0f && signbit(x));
        d[D::device_index(j)] = x;
    }
    ok = __syncthreads_and(ok);
    if (threadIdx.x < uint32_t(D::STRIDE - D::SKIP))
        reinterpret_cast<uint32_t*>(d)[D::SKIP + threadIdx.x] = threadIdx.x == 0 && ok ? 1u : 0u;
}
constexpr uint32_t kRepackThreads = 256;

// Launch-shape variants (warps per block, minimum resident blocks per SM =
// the register cap): the autotuner's search space.
using KernelFn = void (*)(Params);
struct Variant {
    KernelFn fn;
    uint32_t warps, min_blocks;
    uint32_t team = 1;                 // warps per game
    uint32_t games() const { return warps / team; }
};
Variant const kVariants[] = {
    {eval_kernel<4, 3>, 4, 3}, {eval_kernel<4, 4>, 4, 4}, {eval_kernel<4, 5>, 4, 5}, {eval_kernel<4, 6>, 4, 6},
    {eval_kernel<2, 10>, 2, 10}, {eval_kernel<2, 12>, 2, 12},
    // larger blocks (8 and 16 games per block, 256 / 512 threads), same 128-register cap
    {eval_kernel<8, 2>, 8, 2}, {eval_kernel<16, 1>, 16, 1},
    // 20 warps per SM (the 68-word records leave room for them) at a ~100-register cap
    {eval_kernel<10, 2>, 10, 2}, {eval_kernel<20, 1>, 20, 1},
    // two warps per game, 4 games per block (one block per SM, no register cap): batches of at
    // most 4 games per SM run on it by default
    {eval_kernel<8, 1, 0, false, false, 2>, 8, 1, 2},
    // four warps per game (2 games per block): 55 vs 65 us per move at one game per SM, 63 vs 67 at
    // two (eight warps per game measured 69 us: the per-warp top-K and the merges stop the gain)
    {eval_kernel<8, 1, 0, false, false, 4>, 8, 1, 4},
};
// the default variant's hand-off flavour: its launch's tail (at most 4 games per SM) goes to the
// paired kernel
Variant const kHandoffVariant = {eval_kernel<16, 1, 0, false, false, 1, true>, 16, 1};
constexpr int kNumVariants = int(sizeof(kVariants) / sizeof(kVariants[0]));
// the networks a launch can run: v11, or the widened 10 -> H -> H -> 1 for H = 64 or 32
enum NetKind { NET_V11 = 0, NET_W64 = 1, NET_W32 = 2, NUM_NETS = 3 };
constexpr int net_width(int ni) { return ni == NET_W64 ? 64 : ni == NET_W32 ? 32 : 0; }
// dynamic shared memory per warp: its WarpShared block, plus the widened network's hidden-unit buffer
constexpr size_t warp_bytes(int ni) { return sizeof(WarpShared) + size_t(net_width(ni)) * WARP * sizeof(float); }
// the widened networks' launch shapes (more registers per lane than v11): width 64 at 2 blocks
// of 4 warps per SM (255 registers), width 32 at 3
Variant const kWideNet[NUM_NETS] = {{nullptr, 0, 0}, {eval_kernel<4, 2, 64>, 4, 2}, {eval_kernel<4, 3, 32>, 4, 3}};
// the budget-checking flavours (shapes where the extra check spills nothing)
Variant const kBudgetNet[NUM_NETS] = {{eval_kernel<4, 3, 0, true>, 4, 3}, {eval_kernel<4, 2, 64, true>, 4, 2},
                                      {eval_kernel<4, 3, 32, true>, 4, 3}};
// the tracing flavours that record each move's two largest keys (without a time budget)
Variant const kKeysNet[NUM_NETS] = {{eval_kernel<4, 3, 0, false, true>, 4, 3},
                                    {eval_kernel<4, 2, 64, false, true>, 4, 2},
                                    {eval_kernel<4, 3, 32, false, true>, 4, 3}};
constexpr int kNoAllocVariant = 1;   // the allocation-free entry point keeps its fixed 4 x 4 launch shape
constexpr int kSmallVariant = 10;  // the paired kernel: the default for batches of at most 4 games per SM
constexpr int kResumeVariant = kSmallVariant;   // the team kernel that finishes a hand-off's games
constexpr int kTinyVariant = 11;   // teams of four: the default for batches of at most 2 games per SM
constexpr int kDefaultVariant = 7;   // 16 warps, 1 block/SM: the autotuner's pick on the full generation and the stress batch

} // namespace
} // namespace ta3b

// ===================================================================== C ABI ===
using namespace ta3b;

struct ta3b_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int variant = kDefaultVariant;
    uint32_t warps_per_block = 0;
    uint32_t blocks_per_sm = 0;
    uint32_t sms = 0;
    uint32_t grid = 0;
    float* d_w = nullptr;
    size_t cap_w = 0;
    uint64_t* d_seeds = nullptr;
    size_t cap_seeds = 0;
    float* d_score = nullptr;
    uint32_t* d_pieces = nullptr;
    uint32_t* d_lines = nullptr;
    uint32_t* d_evals = nullptr;
    size_t cap_sims = 0;
    uint8_t* d_trace = nullptr;
    size_t cap_trace = 0;
    uint32_t* d_nmoves = nullptr;
    uint32_t* d_board = nullptr;
    size_t cap_tb = 0;
    uint32_t* d_scratch = nullptr;
    uint64_t* d_timing = nullptr;
    size_t cap_timing = 0;
    float* d_wpad = nullptr;          // widened models in their padded device layout
    size_t cap_wpad = 0;
    unsigned long long budget_ns = 0; // per-launch time budget (0 = none)
    uint32_t net_grid[NUM_NETS] = {0, 0, 0};     // widened-network kernels (by NetKind), set up on first use
    uint32_t budget_grid[NUM_NETS] = {0, 0, 0};  // budget flavours (by NetKind), set up on first use
    uint32_t keys_grid[NUM_NETS] = {0, 0, 0};    // key-tracing flavours (by NetKind), set up on first use
    bool auto_small = true;                      // small v11 batches run a team kernel (until a variant is selected)
    uint32_t small_grid = 0;                     // its grid, set up on first use
    uint32_t resume_grid = 0;                    // the hand-off's team kernel's grid
    uint32_t tiny_grid = 0;                      // the teams-of-four kernel's grid (the smallest batches)
    uint32_t test_flags = 0;                     // ta3b_set_test_flags
    bool handoff = true;                         // the default variant hands its launch's tail to the paired kernel
    uint32_t handoff_grid = 0;                   // the hand-off flavour's grid, set up on first use
    Checkpoint* d_ckpt = nullptr;                // the hand-off's checkpoints: one per paired-kernel game slot
    uint32_t ckpt_cap = 0;
    uint64_t* d_keys = nullptr;                  // per move the two largest final keys (tracing)
    size_t cap_keys = 0;
    uint32_t last_grid = 0, last_warps = 0;   // the most recent launch's shape (0: none yet)
    uint32_t last_kernels = 0;                // and how many kernels it launched
    std::string err;
};

namespace {

thread_local std::string g_create_error;

int fail(ta3b_ctx* ctx, int code, std::string const& msg) {
    if (ctx) ctx->err = msg;
    else g_create_error = msg;
    return code;
}

int cuda_fail(ta3b_ctx* ctx, cudaError_t e, char const* what) {
    return fail(ctx, TA3B_ERR_CUDA, std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
}

#define TA3B_CUDA(ctx, call, what)                          \
    do {                                                    \
        cudaError_t const e_ = (call);                      \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

template <class T>
int grow(ta3b_ctx* ctx, T*& ptr, size_t& cap, size_t need, char const* what) {
    if (need <= cap) return TA3B_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    TA3B_CUDA(ctx, cudaMalloc(&ptr, need * sizeof(T)), what);
    cap = need;
    return TA3B_OK;
}

// the network a parameter count selects
int net_of(uint32_t num_params) {
    return num_params == uint32_t(NPARAMS_WIDE) ? NET_W64 : num_params == uint32_t(NPARAMS_WIDE32) ? NET_W32 : NET_V11;
}
uint32_t net_stride(int ni) { return ni == NET_W64 ? Wide64::STRIDE : ni == NET_W32 ? Wide32::STRIDE : NPARAMS; }

// widened models -> their device layout in ctx->d_wpad (grown to fit), on `st`
int repack_models(ta3b_ctx* ctx, int ni, float const* d_src, uint64_t models, cudaStream_t st) {
    if (int rc = grow(ctx, ctx->d_wpad, ctx->cap_wpad, models * net_stride(ni), "alloc padded weights")) return rc;
    if (ni == NET_W64)
        repack_wide_kernel<64><<<uint32_t(models), kRepackThreads, 0, st>>>(d_src, uint32_t(models), ctx->d_wpad);
    else
        repack_wide_kernel<32><<<uint32_t(models), kRepackThreads, 0, st>>>(d_src, uint32_t(models), ctx->d_wpad);
    TA3B_CUDA(ctx, cudaGetLastError(), "repack widened weights");
    return TA3B_OK;
}

int check_sizes(ta3b_ctx* ctx, uint32_t num_islands, uint32_t models_per_island, uint32_t num_params,
                uint32_t num_games) {
    if (!ctx) return fail(ctx, TA3B_ERR_ARG, "null context");
    if (num_params != NPARAMS && num_params != uint32_t(NPARAMS_WIDE) && num_params != uint32_t(NPARAMS_WIDE32))
        return fail(ctx, TA3B_ERR_ARG, "num_params must be " + std::to_string(NPARAMS) + " (v11), " +
                                           std::to_string(NPARAMS_WIDE) + " (10 -> 64 -> 64 -> 1) or " +
                                           std::to_string(NPARAMS_WIDE32) + " (10 -> 32 -> 32 -> 1)");
    uint64_t const sims = uint64_t(num_islands) * models_per_island * num_games;
    if (sims > kMaxSims) return fail(ctx, TA3B_ERR_ARG, "too many sims in one batch (at most 2^32 - 1)");
    return TA3B_OK;
}

// The widened kernels read each model's 19.7 KB of weights through L1, which
// shares its on-chip memory with shared memory: ask for just the shared memory
// that min_blocks resident blocks need, so the rest stays L1 (a 20k-sim
// generation on B200: 24.7 s with the maximum shared-memory split, 20.6 s with
// this one). Handing each SM its own contiguous range of sims, so that its warps
// share models, measured slower (26.1 s) than the single queue.
int set_min_carveout(ta3b_ctx* ctx, Variant const& v, size_t dyn) {
    int per_sm = 0, reserved = 0;
    TA3B_CUDA(ctx, cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device), "smem per SM");
    TA3B_CUDA(ctx, cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, ctx->device),
              "reserved smem per block");
    cudaFuncAttributes fa{};
    TA3B_CUDA(ctx, cudaFuncGetAttributes(&fa, v.fn), "kernel attributes");
    size_t const need = size_t(v.min_blocks) * (dyn + fa.sharedSizeBytes + size_t(reserved));
    int const pct = per_sm > 0 ? int((need * 100 + size_t(per_sm) - 1) / size_t(per_sm)) : 100;
    TA3B_CUDA(ctx, cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct < 100 ? pct : 100),
              "smem carveout");
    return TA3B_OK;
}

// shared-memory limits, carveout and resident grid of one widened or budget kernel
int setup_kernel(ta3b_ctx* ctx, Variant const& v, int ni, uint32_t& grid_out, char const* what) {
    size_t const dyn = v.warps * warp_bytes(ni);
    TA3B_CUDA(ctx, cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)), "dynamic smem size");
    if (ni != NET_V11) {
        if (int rc = set_min_carveout(ctx, v, dyn)) return rc;
    } else {
        TA3B_CUDA(ctx, cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            cudaSharedmemCarveoutMaxShared), "smem carveout");
    }
    int per_sm = 0;
    TA3B_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.warps * 32, dyn), "occupancy");
    if (ni != NET_V11 && per_sm < int(v.min_blocks)) {   // the split chosen leaves too little shared memory
        TA3B_CUDA(ctx, cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            cudaSharedmemCarveoutMaxShared), "smem carveout");
        TA3B_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.warps * 32, dyn), "occupancy");
    }
    if (per_sm < 1) return fail(ctx, TA3B_ERR_CUDA, std::string(what) + " does not fit on an SM");
    grid_out = ctx->sms * uint32_t(per_sm);
    return TA3B_OK;
}

int launch(ta3b_ctx* ctx, Params const& prm, cudaStream_t st, int ni = NET_V11) {
    if (prm.total_sims == 0) return TA3B_OK;
    if (ni != NET_V11 && !ctx->net_grid[ni])
        if (int rc = setup_kernel(ctx, kWideNet[ni], ni, ctx->net_grid[ni], "widened kernel")) return rc;
    bool const keys = prm.keys != nullptr;
    bool const budget = ctx->budget_ns != 0 && !keys;
    if (budget && !ctx->budget_grid[ni])
        if (int rc = setup_kernel(ctx, kBudgetNet[ni], ni, ctx->budget_grid[ni], "budget kernel")) return rc;
    if (keys && !ctx->keys_grid[ni])
        if (int rc = setup_kernel(ctx, kKeysNet[ni], ni, ctx->keys_grid[ni], "key-tracing kernel")) return rc;
    TA3B_CUDA(ctx, cudaMemsetAsync(prm.scratch, 0, kScratchBytes, st), "reset work queue");
    // with a time budget the budget-checking flavour runs, with key tracing the tracing flavour
    // (which runs without the budget); each has its own fixed launch shape
    // unless a variant was selected, a v11 batch of at most 4 games per SM runs on the paired kernel
    // (two warps per game), whose moves take 0.62x the single-warp kernel's time at that load, and
    // one of at most 2 games per SM on teams of four warps (0.53x)
    Variant const& small = kVariants[kSmallVariant];
    Variant const& tiny = kVariants[kTinyVariant];
    bool const auto_small = ctx->auto_small && ni == NET_V11 && !keys && !budget;
    bool const use_tiny = auto_small && prm.total_sims <= ctx->sms * tiny.games();
    bool const use_small = auto_small && !use_tiny && prm.total_sims <= ctx->sms * small.games();
    if (use_small && !ctx->small_grid)
        if (int rc = setup_kernel(ctx, small, NET_V11, ctx->small_grid, "paired kernel")) return rc;
    if (use_tiny && !ctx->tiny_grid)
        if (int rc = setup_kernel(ctx, tiny, NET_V11, ctx->tiny_grid, "teams-of-four kernel")) return rc;
    Variant const* const v = keys     ? &kKeysNet[ni]
                             : budget ? &kBudgetNet[ni]
                             : ni != NET_V11 ? &kWideNet[ni]
                             : use_tiny ? &tiny : use_small ? &small : &kVariants[ctx->variant];
    uint32_t const warps = v->warps, games = v->games();
    uint32_t const max_grid = keys     ? ctx->keys_grid[ni]
                              : budget ? ctx->budget_grid[ni]
                              : ni != NET_V11 ? ctx->net_grid[ni]
                              : use_tiny ? ctx->tiny_grid : use_small ? ctx->small_grid : ctx->grid;
    // a batch that one block per SM can hold is spread over every SM, one block each (a game runs
    // faster on an SM it shares with fewer others), rather than packed into the fewest blocks
    uint32_t const sims = prm.total_sims;
    bool const spread = sims < ctx->sms * games && ctx->sms <= max_grid;
    uint32_t const need_blocks = (sims + games - 1) / games;
    uint32_t const grid = spread ? (sims < ctx->sms ? (sims ? sims : 1u) : ctx->sms)
                                 : (need_blocks < max_grid ? need_blocks : max_grid);
    Params p2 = prm;
    p2.warps_active = spread ? (sims + grid - 1) / grid * (warps / games) : 0u;
    p2.budget_ns = ctx->budget_ns;
    p2.test_flags = ctx->test_flags;
    // the default variant on a full batch: its launch's tail (at most one paired-kernel slot's worth
    // of games still playing) is checkpointed and finished by the paired kernel, two warps a game
    bool const handoff = ctx->handoff && ctx->d_ckpt && v == &kVariants[kDefaultVariant] && !spread;
    if (handoff) {
        if (!ctx->handoff_grid)
            if (int rc = setup_kernel(ctx, kHandoffVariant, NET_V11, ctx->handoff_grid, "hand-off kernel")) return rc;
        Variant const& resume = kVariants[kResumeVariant];
        if (!ctx->resume_grid)
            if (int rc = setup_kernel(ctx, resume, NET_V11, ctx->resume_grid, "hand-off's team kernel")) return rc;
        p2.ckpt = ctx->d_ckpt;
        p2.ckpt_cap = ctx->ckpt_cap;
        p2.handoff_at = ctx->ckpt_cap < ctx->resume_grid * resume.games() ? ctx->ckpt_cap : ctx->resume_grid * resume.games();
        kHandoffVariant.fn<<<grid, warps * 32, warps * warp_bytes(ni), st>>>(p2);
        TA3B_CUDA(ctx, cudaGetLastError(), "kernel launch");
        Params p3 = p2;
        p3.resume = 1;
        p3.warps_active = 0;
        resume.fn<<<ctx->resume_grid, resume.warps * 32, resume.warps * warp_bytes(NET_V11), st>>>(p3);
    } else {
        v->fn<<<grid, warps * 32, warps * warp_bytes(ni), st>>>(p2);
    }
    TA3B_CUDA(ctx, cudaGetLastError(), "kernel launch");
    ctx->last_grid = grid;
    ctx->last_warps = warps;
    ctx->last_kernels = handoff ? 2u : 1u;
    return TA3B_OK;
}

int status_code(ta3b_ctx* ctx, uint32_t status);

int read_status(ta3b_ctx* ctx) {
    uint32_t status = 0;
    TA3B_CUDA(ctx, cudaMemcpyAsync(&status, ctx->d_scratch + kStatusWord, sizeof status, cudaMemcpyDeviceToHost,
                                   ctx->stream), "read status");
    TA3B_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "kernel run");
    return status_code(ctx, status);
}

// the call's result for a status word: bit 1 = the time budget ran out, any other bit = a device error
int status_code(ta3b_ctx* ctx, uint32_t status) {
    if (status & ~2u) return fail(ctx, TA3B_ERR_DEVICE, "kernel reported status " + std::to_string(status));
    if (status & 2u)
        return fail(ctx, TA3B_ERR_TIMEOUT, "time budget exceeded: the launch stopped early, results are incomplete");
    return TA3B_OK;
}

int host_eval(ta3b_ctx* ctx, float const* weights, uint32_t num_islands, uint32_t mpi, uint32_t num_params,
              uint64_t const* seeds, uint32_t num_games, uint32_t max_moves, float* score_out, uint32_t* pieces_out,
              uint32_t* lines_out, uint32_t* evals_out, uint8_t* trace_out, uint32_t* nmoves_out,
              uint32_t* board_out, uint64_t* timing_out = nullptr, uint64_t* keys_out = nullptr) {
    if (int rc = check_sizes(ctx, num_islands, mpi, num_params, num_games)) return rc;
    uint64_t const models = uint64_t(num_islands) * mpi;
    uint64_t const sims = models * num_games;
    if (sims == 0) return TA3B_OK;
    if (!weights || !seeds || !score_out) return fail(ctx, TA3B_ERR_ARG, "null weights / seeds / score_out");
    TA3B_CUDA(ctx, cudaSetDevice(ctx->device), "set device");
    if (int rc = grow(ctx, ctx->d_w, ctx->cap_w, models * num_params, "alloc weights")) return rc;
    if (int rc = grow(ctx, ctx->d_seeds, ctx->cap_seeds, uint64_t(num_islands) * num_games, "alloc seeds")) return rc;
    if (ctx->cap_sims < sims) {
        size_t c = ctx->cap_sims;
        if (int rc = grow(ctx, ctx->d_score, c, sims, "alloc score")) return rc;
        c = ctx->cap_sims;
        if (int rc = grow(ctx, ctx->d_pieces, c, sims, "alloc pieces")) return rc;
        c = ctx->cap_sims;
        if (int rc = grow(ctx, ctx->d_lines, c, sims, "alloc lines")) return rc;
        c = ctx->cap_sims;
        if (int rc = grow(ctx, ctx->d_evals, c, sims, "alloc evals")) return rc;
        ctx->cap_sims = sims;
    }
    bool const tracing = trace_out || nmoves_out || board_out || keys_out;
    if (keys_out)
        if (int rc = grow(ctx, ctx->d_keys, ctx->cap_keys, sims * max_moves * 2 + 2, "alloc keys")) return rc;
    if (timing_out)
        if (int rc = grow(ctx, ctx->d_timing, ctx->cap_timing, 2 * sims, "alloc timing")) return rc;
    if (tracing) {
        if (int rc = grow(ctx, ctx->d_trace, ctx->cap_trace, sims * max_moves * 3 + 1, "alloc trace")) return rc;
        if (ctx->cap_tb < sims) {
            size_t c = ctx->cap_tb;
            if (int rc = grow(ctx, ctx->d_nmoves, c, sims, "alloc n_moves")) return rc;
            c = ctx->cap_tb;
            if (int rc = grow(ctx, ctx->d_board, c, sims * W, "alloc boards")) return rc;
            ctx->cap_tb = sims;
        }
    }
    int const ni = net_of(num_params);
    bool const wide = ni != NET_V11;
    if (wide) {   // the models as given (d_w), then their device layout (d_wpad)
        TA3B_CUDA(ctx, cudaMemcpyAsync(ctx->d_w, weights, models * num_params * sizeof(float), cudaMemcpyHostToDevice,
                                       ctx->stream), "copy weights");
        if (int rc = repack_models(ctx, ni, ctx->d_w, models, ctx->stream)) return rc;
    } else {
        TA3B_CUDA(ctx, cudaMemcpyAsync(ctx->d_w, weights, models * num_params * sizeof(float),
                                       cudaMemcpyHostToDevice, ctx->stream), "copy weights");
    }
    TA3B_CUDA(ctx, cudaMemcpyAsync(ctx->d_seeds, seeds, uint64_t(num_islands) * num_games * sizeof(uint64_t),
                                   cudaMemcpyHostToDevice, ctx->stream), "copy seeds");
    Params prm{};
    prm.weights = wide ? ctx->d_wpad : ctx->d_w;
    prm.seeds = ctx->d_seeds;
    prm.score = ctx->d_score;
    prm.pieces = ctx->d_pieces;
    prm.lines = ctx->d_lines;
    prm.evals = ctx->d_evals;
    prm.trace = tracing ? ctx->d_trace : nullptr;
    prm.n_moves = tracing ? ctx->d_nmoves : nullptr;
    prm.board_out = tracing ? ctx->d_board : nullptr;
    prm.scratch = ctx->d_scratch;
    prm.timing = timing_out ? reinterpret_cast<unsigned long long*>(ctx->d_timing) : nullptr;
    prm.keys = keys_out ? reinterpret_cast<unsigned long long*>(ctx->d_keys) : nullptr;
    prm.num_games = num_games;
    prm.models_per_island = mpi;
    prm.max_moves = max_moves;
    prm.total_sims = uint32_t(sims);
    if (int rc = launch(ctx, prm, ctx->stream, ni)) return rc;
    TA3B_CUDA(ctx, cudaMemcpyAsync(score_out, ctx->d_score, sims * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
              "copy score");
    if (pieces_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(pieces_out, ctx->d_pieces, sims * 4, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy pieces");
    if (lines_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(lines_out, ctx->d_lines, sims * 4, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy lines");
    if (evals_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(evals_out, ctx->d_evals, sims * 4, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy evals");
    if (trace_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(trace_out, ctx->d_trace, sims * max_moves * 3, cudaMemcpyDeviceToHost,
                                       ctx->stream), "copy trace");
    if (nmoves_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(nmoves_out, ctx->d_nmoves, sims * 4, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy n_moves");
    if (board_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(board_out, ctx->d_board, sims * W * 4, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy boards");
    if (timing_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(timing_out, ctx->d_timing, sims * 16, cudaMemcpyDeviceToHost, ctx->stream),
                  "copy timing");
    if (keys_out)
        TA3B_CUDA(ctx, cudaMemcpyAsync(keys_out, ctx->d_keys, sims * max_moves * 16, cudaMemcpyDeviceToHost,
                                       ctx->stream), "copy keys");
    return read_status(ctx);
}

int select_variant(ta3b_ctx* ctx, int v) {
    if (v < 0 || v >= kNumVariants) return fail(ctx, TA3B_ERR_ARG, "variant out of range");
    TA3B_CUDA(ctx, cudaSetDevice(ctx->device), "set device");
    size_t const dyn = kVariants[v].warps * sizeof(WarpShared);
    TA3B_CUDA(ctx, cudaFuncSetAttribute(kVariants[v].fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)),
              "dynamic smem size");
    TA3B_CUDA(ctx, cudaFuncSetAttribute(kVariants[v].fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        cudaSharedmemCarveoutMaxShared), "smem carveout");
    int per_sm = 0;
    TA3B_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kVariants[v].fn, kVariants[v].warps * 32, dyn),
              "occupancy");
    if (per_sm < 1) return fail(ctx, TA3B_ERR_CUDA, "kernel variant does not fit on an SM");
    ctx->variant = v;
    ctx->auto_small = false;
    ctx->warps_per_block = kVariants[v].warps;
    ctx->blocks_per_sm = uint32_t(per_sm);
    ctx->grid = ctx->sms * ctx->blocks_per_sm;
    return TA3B_OK;
}

} // namespace

extern "C" {

ta3b_ctx* ta3b_create(ta3b_config const* cfg) {
    ta3b_config const c = cfg ? *cfg : ta3b_config{0, 0, 0};
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (c.device < 0 || c.device >= n) {
        g_create_error = "device ordinal out of range";
        return nullptr;
    }
    cudaDeviceProp prop{};
    if ((e = cudaGetDeviceProperties(&prop, c.device)) != cudaSuccess) {
        g_create_error = std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (prop.major != 10) {
        g_create_error = "this build targets sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                         std::to_string(prop.minor);
        return nullptr;
    }
    auto* ctx = new ta3b_ctx();
    ctx->device = c.device;
    ctx->sms = uint32_t(prop.multiProcessorCount);
    if (cudaSetDevice(c.device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_scratch, kScratchBytes) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_scratch, 0, kScratchBytes, ctx->stream) != cudaSuccess ||   // (the context's stream
        cudaStreamSynchronize(ctx->stream) != cudaSuccess ||                              // orders every later use)
        cudaMalloc(&ctx->d_ckpt, size_t(ctx->sms) * kVariants[kResumeVariant].games() * sizeof(Checkpoint)) != cudaSuccess) {
        g_create_error = std::string("context setup: ") + cudaGetErrorString(cudaGetLastError());
        ta3b_destroy(ctx);
        return nullptr;
    }
    ctx->ckpt_cap = ctx->sms * kVariants[kResumeVariant].games();
    int v = kDefaultVariant;
    if (c.warps_per_block || c.blocks_per_sm) {
        v = -1;
        for (int i = 0; i < kNumVariants; ++i)
            if (kVariants[i].team == 1 && (!c.warps_per_block || kVariants[i].warps == c.warps_per_block) &&
                (!c.blocks_per_sm || kVariants[i].min_blocks == c.blocks_per_sm)) {
                v = i;
                break;
            }
        if (v < 0) {
            g_create_error = "no kernel variant with that warps_per_block / blocks_per_sm (see ta3b_variant_info)";
            ta3b_destroy(ctx);
            return nullptr;
        }
    }
    if (select_variant(ctx, v) != TA3B_OK) {
        g_create_error = ctx->err;
        ta3b_destroy(ctx);
        return nullptr;
    }
    ctx->auto_small = !(c.warps_per_block || c.blocks_per_sm);   // a requested shape is kept for every batch
    return ctx;
}

void ta3b_destroy(ta3b_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    void* bufs[] = {ctx->d_w, ctx->d_seeds, ctx->d_score, ctx->d_pieces, ctx->d_lines, ctx->d_evals,
                    ctx->d_trace, ctx->d_nmoves, ctx->d_board, ctx->d_scratch, ctx->d_timing, ctx->d_wpad,
                    ctx->d_keys, ctx->d_ckpt};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

char const* ta3b_last_error(ta3b_ctx const* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int ta3b_eval(ta3b_ctx* ctx, float const* weights, uint32_t num_models, uint32_t num_params, uint64_t const* seeds,
              uint32_t num_games, uint32_t max_moves, float* score_out, uint32_t* pieces_out, uint32_t* lines_out) {
    return host_eval(ctx, weights, 1, num_models, num_params, seeds, num_games, max_moves, score_out, pieces_out,
                     lines_out, nullptr, nullptr, nullptr, nullptr);
}

int ta3b_eval_islands(ta3b_ctx* ctx, float const* weights, uint32_t num_islands, uint32_t models_per_island,
                      uint32_t num_params, uint64_t const* seeds, uint32_t num_games, uint32_t max_moves,
                      float* score_out, uint32_t* pieces_out, uint32_t* lines_out) {
    return host_eval(ctx, weights, num_islands, models_per_island, num_params, seeds, num_games, max_moves, score_out,
                     pieces_out, lines_out, nullptr, nullptr, nullptr, nullptr);
}

int ta3b_eval_trace(ta3b_ctx* ctx, float const* weights, uint32_t num_models, uint32_t num_params,
                    uint64_t const* seeds, uint32_t num_games, uint32_t max_moves, float* score_out,
                    uint32_t* pieces_out, uint32_t* lines_out, uint32_t* evals_out, uint8_t* trace_out,
                    uint32_t* n_moves_out, uint32_t* board_out, uint64_t* keys_out) {
    return host_eval(ctx, weights, 1, num_models, num_params, seeds, num_games, max_moves, score_out, pieces_out,
                     lines_out, evals_out, trace_out, n_moves_out, board_out, nullptr, keys_out);
}

int ta3b_eval_timed(ta3b_ctx* ctx, float const* weights, uint32_t num_islands, uint32_t models_per_island,
                    uint32_t num_params, uint64_t const* seeds, uint32_t num_games, uint32_t max_moves,
                    float* score_out, uint32_t* pieces_out, uint32_t* evals_out, uint64_t* timing_out) {
    return host_eval(ctx, weights, num_islands, models_per_island, num_params, seeds, num_games, max_moves, score_out,
                     pieces_out, nullptr, evals_out, nullptr, nullptr, nullptr, timing_out);
}

int ta3b_eval_device(ta3b_ctx* ctx, float const* d_weights, uint32_t num_islands, uint32_t models_per_island,
                     uint32_t num_params, uint64_t const* d_seeds, uint32_t num_games, uint32_t max_moves,
                     float* d_score, uint32_t* d_pieces, uint32_t* d_lines, uint32_t* d_evals, void* stream) {
    if (int rc = check_sizes(ctx, num_islands, models_per_island, num_params, num_games)) return rc;
    uint64_t const sims = uint64_t(num_islands) * models_per_island * num_games;
    if (sims == 0) return TA3B_OK;
    if (!d_weights || !d_seeds || !d_score) return fail(ctx, TA3B_ERR_ARG, "null device pointer");
    cudaStream_t const st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    int const ni = net_of(num_params);
    bool const wide = ni != NET_V11;
    if (wide)   // the padded copy (allocated on the first widened call of this size)
        if (int rc = repack_models(ctx, ni, d_weights, uint64_t(num_islands) * models_per_island, st)) return rc;
    Params prm{};
    prm.weights = wide ? ctx->d_wpad : d_weights;
    prm.seeds = d_seeds;
    prm.score = d_score;
    prm.pieces = d_pieces;
    prm.lines = d_lines;
    prm.evals = d_evals;
    prm.scratch = ctx->d_scratch;
    prm.num_games = num_games;
    prm.models_per_island = models_per_island;
    prm.max_moves = max_moves;
    prm.total_sims = uint32_t(sims);
    return launch(ctx, prm, st, ni);
}

int ta3b_simulate_seeds(uint64_t seed, uint32_t games, uint64_t* seeds_out) {
    if (games && !seeds_out) return TA3B_ERR_ARG;
    uint64_t s[4];
    for (int i = 0; i < 4; ++i) {
        seed += 0x9e3779b97f4a7c15ULL;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        s[i] = z ^ (z >> 31);
    }
    for (uint32_t g = 0; g < games; ++g) {
        uint64_t const r = ((s[1] * 5) << 7 | (s[1] * 5) >> 57) * 9;
        uint64_t const t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = (s[3] << 45) | (s[3] >> 19);
        seeds_out[g] = r;
    }
    return TA3B_OK;
}

int ta3b_core_selftest(uint32_t const* recs, uint32_t num_recs, uint32_t const* cand, uint32_t n, float const* w97,
                       float* fast_v, int* fast_st, float* full_v, int* full_legal, float* dbg32) {
    if (!recs || !cand || !w97 || !fast_v || !fast_st || !full_v || !full_legal) return TA3B_ERR_ARG;
    if (n == 0) return TA3B_OK;
    void* d[8] = {};
    size_t const sz[8] = {size_t(num_recs) * REC_WORDS * 4, size_t(n) * 4, NPARAMS * 4, size_t(n) * 4, size_t(n) * 4,
                          size_t(n) * 4, size_t(n) * 4, dbg32 ? size_t(n) * 32 * 4 : 4};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 8 && e == cudaSuccess; ++k) e = cudaMalloc(&d[k], sz[k]);
    if (e == cudaSuccess) e = cudaMemcpy(d[0], recs, sz[0], cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d[1], cand, sz[1], cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d[2], w97, sz[2], cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        core_selftest_kernel<<<(n + 127) / 128, 128>>>(static_cast<uint32_t*>(d[0]), static_cast<uint32_t*>(d[1]), n,
                                                        static_cast<float*>(d[2]), static_cast<float*>(d[3]),
                                                        static_cast<int*>(d[4]), static_cast<float*>(d[5]),
                                                        static_cast<int*>(d[6]),
                                                        dbg32 ? static_cast<float*>(d[7]) : nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(fast_v, d[3], sz[3], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(fast_st, d[4], sz[4], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(full_v, d[5], sz[5], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(full_legal, d[6], sz[6], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && dbg32) e = cudaMemcpy(dbg32, d[7], sz[7], cudaMemcpyDeviceToHost);
    for (void* q : d)
        if (q) cudaFree(q);
    if (e != cudaSuccess) {
        g_create_error = std::string("core selftest: ") + cudaGetErrorString(e);
        return TA3B_ERR_CUDA;
    }
    return TA3B_OK;
}

int ta3b_set_test_flags(ta3b_ctx* ctx, uint32_t flags) {
    if (!ctx || (flags & ~1u)) return ctx ? fail(ctx, TA3B_ERR_ARG, "unknown test flag") : TA3B_ERR_ARG;
    ctx->test_flags = flags;
    return TA3B_OK;
}

int ta3b_set_tail_handoff(ta3b_ctx* ctx, int on) {
    if (!ctx) return TA3B_ERR_ARG;
    ctx->handoff = on != 0;
    return TA3B_OK;
}

int ta3b_handoff_info(ta3b_ctx* ctx, uint32_t* games_out) {
    if (!ctx || !games_out) return TA3B_ERR_ARG;
    uint32_t n = 0;
    TA3B_CUDA(ctx, cudaMemcpyAsync(&n, ctx->d_scratch + kCkptCountWord, sizeof n, cudaMemcpyDeviceToHost, ctx->stream),
              "read hand-off count");
    TA3B_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "read hand-off count");
    *games_out = n < ctx->ckpt_cap ? n : ctx->ckpt_cap;
    return TA3B_OK;
}

int ta3b_num_variants(void) { return kNumVariants; }

int ta3b_variant_warps_per_game(int variant) {
    if (variant < 0 || variant >= kNumVariants) return -1;
    return int(kVariants[variant].team);
}

int ta3b_variant_info(int variant, uint32_t* warps_per_block, uint32_t* min_blocks_per_sm) {
    if (variant < 0 || variant >= kNumVariants) return TA3B_ERR_ARG;
    if (warps_per_block) *warps_per_block = kVariants[variant].warps;
    if (min_blocks_per_sm) *min_blocks_per_sm = kVariants[variant].min_blocks;
    return TA3B_OK;
}

int ta3b_set_time_budget(ta3b_ctx* ctx, double seconds) {
    if (!ctx) return TA3B_ERR_ARG;
    if (!(seconds >= 0.0) || seconds > 1.0e6) return fail(ctx, TA3B_ERR_ARG, "time budget must be in [0, 1e6] s");
    ctx->budget_ns = static_cast<unsigned long long>(seconds * 1.0e9);
    return TA3B_OK;
}

int ta3b_select_variant(ta3b_ctx* ctx, int variant) {
    if (!ctx) return TA3B_ERR_ARG;
    return select_variant(ctx, variant);
}

int ta3b_launch_info(ta3b_ctx const* ctx, uint32_t* grid, uint32_t* warps_per_block, uint32_t* sms,
                     uint32_t* kernels) {
    if (!ctx) return TA3B_ERR_ARG;
    if (grid) *grid = ctx->last_grid ? ctx->last_grid : ctx->grid;
    if (warps_per_block) *warps_per_block = ctx->last_grid ? ctx->last_warps : ctx->warps_per_block;
    if (sms) *sms = ctx->sms;
    if (kernels) *kernels = ctx->last_kernels;
    return TA3B_OK;
}

int ta3b_device_status(ta3b_ctx* ctx, uint32_t* status_out) {
    if (!ctx) return TA3B_ERR_ARG;
    TA3B_CUDA(ctx, cudaSetDevice(ctx->device), "set device");
    uint32_t status = 0;
    TA3B_CUDA(ctx, cudaMemcpyAsync(&status, ctx->d_scratch + kStatusWord, sizeof status, cudaMemcpyDeviceToHost,
                                   ctx->stream), "read status");
    TA3B_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "read status");
    if (status_out) *status_out = status;
    return status_code(ctx, status);
}

} // extern "C"

// ============================================ allocation-free evaluation ===
// Some hosts cannot call cudaMalloc where they evaluate: a framework whose own
// pooling allocator owns all device memory (raw cudaMalloc/cudaFree calls
// bypass its accounting and can fragment or exhaust its pool), or a latency-
// critical scheduler thread that must not pay cudaMalloc/cudaFree's implicit
// device-wide synchronisation. ta3b_eval_device_noalloc serves them: it creates
// no context and allocates nothing. The caller passes device inputs and
// outputs; the only scratch the evaluation kernel needs -- its 64-bit work-queue
// ticket (words 0-1) and error status word (word 2) -- lives in the file-scope
// array below, which every GPU that loads this library holds until the process
// exits.
namespace {

constexpr uint32_t kNoAllocScratchWords = 64;                 // 256 bytes; words 0-2 used
constexpr uint64_t kNoAllocMaxSims = kMaxSims;                // the 64-bit ticket cannot wrap
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchWords];
static_assert(kScratchBytes <= sizeof(g_noalloc_scratch), "the work-queue words fit the static array");

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
    uint32_t* scratch;   // device address of g_noalloc_scratch on this device
    uint32_t grid, sms;
    bool ready;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

} // namespace

extern "C" int ta3b_eval_device_noalloc(float const* d_weights, uint32_t num_islands, uint32_t models_per_island,
                                        uint32_t num_params, uint64_t const* d_seeds, uint32_t num_games,
                                        uint32_t max_moves, float* d_score, uint32_t* d_pieces, uint32_t* d_lines,
                                        uint32_t* d_evals, void* stream, char const** error_out) {
    auto fail_static = [&](int code, char const* msg) {
        if (error_out) *error_out = msg;
        return code;
    };
    if (error_out) *error_out = "";
    if (num_params != NPARAMS) return fail_static(TA3B_ERR_ARG, "num_params must be 97 (v11 value model)");
    uint64_t const sims = uint64_t(num_islands) * models_per_island * num_games;
    if (sims > kNoAllocMaxSims)
        return fail_static(TA3B_ERR_ARG, "too many sims for the allocation-free path (at most 2^32 - 1 per call)");
    if (sims == 0) return TA3B_OK;
    if (!d_weights || !d_seeds || !d_score) return fail_static(TA3B_ERR_ARG, "null device pointer");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
        return fail_static(TA3B_ERR_CUDA, "cudaGetDevice failed or device ordinal too large");
    Variant const& var = kVariants[kNoAllocVariant];
    size_t const dyn = var.warps * sizeof(WarpShared);
    {
        // once per device, with that device current: resolve the scratch array's
        // device address (its host-side name is only a stand-in) and set the
        // kernel's shared-memory limit
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoAllocDevice& d = g_noalloc_dev[dev];
        if (!d.ready) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
                return fail_static(TA3B_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
            if (cudaFuncSetAttribute(var.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)) != cudaSuccess)
                return fail_static(TA3B_ERR_CUDA, "cudaFuncSetAttribute failed");
            int sms = 0, per_sm = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, var.fn, int(var.warps * 32), dyn) != cudaSuccess ||
                per_sm < 1)
                return fail_static(TA3B_ERR_CUDA, "occupancy query failed");
            d.scratch = static_cast<uint32_t*>(ptr);
            d.grid = uint32_t(sms) * uint32_t(per_sm);
            d.sms = uint32_t(sms);
            d.ready = true;
        }
    }
    NoAllocDevice const& d = g_noalloc_dev[dev];
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: the ticket and status must start at zero
    if (cudaMemsetAsync(d.scratch, 0, kScratchBytes, st) != cudaSuccess)
        return fail_static(TA3B_ERR_CUDA, "clearing the scratch array failed");
    Params prm{};
    prm.weights = d_weights;
    prm.seeds = d_seeds;
    prm.score = d_score;
    prm.pieces = d_pieces;
    prm.lines = d_lines;
    prm.evals = d_evals;
    prm.scratch = d.scratch;
    prm.num_games = num_games;
    prm.models_per_island = models_per_island;
    prm.max_moves = max_moves;
    prm.total_sims = uint32_t(sims);
    // a batch that one block per SM can hold is spread over every SM (as on the context path)
    uint32_t const need = uint32_t((sims + var.warps - 1) / var.warps);
    bool const spread = sims < uint64_t(d.sms) * var.warps;
    uint32_t const grid = spread ? uint32_t(sims < d.sms ? sims : d.sms) : (need < d.grid ? need : d.grid);
    if (spread) prm.warps_active = uint32_t((sims + grid - 1) / grid);
    var.fn<<<grid, var.warps * 32, dyn, st>>>(prm);
    if (cudaGetLastError() != cudaSuccess) return fail_static(TA3B_ERR_CUDA, "kernel launch failed");
    return TA3B_OK;
}

// The status word the most recent allocation-free call on the current device left
// in the static array: copied on `stream` (NULL = legacy default stream) after the
// work already queued there, which must include that call. Allocates nothing.
extern "C" int ta3b_noalloc_status(void* stream, uint32_t* status_out, char const** error_out) {
    if (error_out) *error_out = "";
    if (!status_out) {
        if (error_out) *error_out = "null status_out";
        return TA3B_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        if (error_out) *error_out = "cudaGetDevice failed or device ordinal too large";
        return TA3B_ERR_CUDA;
    }
    uint32_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (g_noalloc_dev[dev].ready) scratch = g_noalloc_dev[dev].scratch;
    }
    if (!scratch) {
        if (error_out) *error_out = "no allocation-free evaluation has run on this device";
        return TA3B_ERR_ARG;
    }
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    uint32_t status = 0;
    if (cudaMemcpyAsync(&status, scratch + kStatusWord, sizeof status, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        if (error_out) *error_out = "reading the status word failed";
        return TA3B_ERR_CUDA;
    }
    *status_out = status;
    if (status) {
        if (error_out) *error_out = "the kernel reported a device error status";
        return TA3B_ERR_DEVICE;
    }
    return TA3B_OK;
}
