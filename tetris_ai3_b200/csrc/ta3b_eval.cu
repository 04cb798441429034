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
// Lanes stride the flattened (parent, child list, placement) space of a level;
// every candidate is one fused apply (fit + lock + line clear) + v11 features
// + FP32 MLP, evaluated in the reference's operation order. The top-K of a
// level is a warp-distributed sorted list (lane i holds the i-th best packed
// key) maintained with ballots and shuffles, so level scores never touch
// memory. Kept frontier boards live in per-warp shared memory; nothing in the
// move loop synchronises more than one warp.
#include "ta3b.h"
#include "tables.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

namespace ta3b {
namespace {

constexpr int WARP = 32;

// ---------------------------------------------------------------- tables ---
// Placement LUT packed one u32 per placement: cols (16) | col0 (4) << 16 |
// orientation (2) << 20 | (x + 2) (4) << 24.
__host__ __device__ constexpr uint32_t pack_place(Place p) {
    return uint32_t(p.cols) | (uint32_t(p.col0) << 16) | (uint32_t(p.orient) << 20) | (uint32_t(p.x + 2) << 24);
}

struct DevTables {
    uint32_t place[NPIECE][MP];
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
        for (int i = 0; i < MP; ++i) d.place[p][i] = i < TABLES.nplace[p] ? pack_place(TABLES.place[p][i]) : 0u;
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

// ------------------------------------------------------------ bit helpers ---
__device__ __forceinline__ int ctz32(uint32_t v) { return __ffs(int(v)) - 1; }   // v != 0
__device__ __forceinline__ int column_top(uint32_t col) { return ctz32(col | FLOOR); }

__device__ __forceinline__ uint32_t ordered_bits(float v) {                  // beam.hpp:204-207
    uint32_t const u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_bits_inv(uint32_t s) {              // beam.hpp:209-211
    return __uint_as_float((s & 0x80000000u) ? (s ^ 0x80000000u) : ~s);
}
__device__ __forceinline__ uint32_t clear_bump(int cleared) {                // model_defs.hpp:177-183
    return cleared == 0 ? 0u : 1u << (8 * (cleared - 1));
}

// remove the rows flagged in `full` from one column, survivors drop down (board2.hpp:218-234)
__device__ __forceinline__ uint32_t clear_rows(uint32_t col, uint32_t full) {
    while (full) {
        uint32_t const row = full & (~full + 1u);
        col = ((col & (row - 1u)) << 1) | (col & ~((row << 1) - 1u));
        full ^= row;
    }
    return col;
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

// hard drop at window x-origin x in orientation o; returns rows cleared or -1 on top-out
__device__ int engine_place(Engine& e, int o, int x) {                       // tetris_engine.hpp:137-146
    uint32_t const p = e.queue[0];
    uint32_t const cols = c_tables.shape_cols[p][o];
    int const col0 = x + c_tables.shape_left[p][o];
    int drop = H;
    for (int i = 0; i < 4; ++i) {                                            // board2.hpp:262-275
        uint32_t const nib = (cols >> (4 * i)) & 0xFu;
        if (nib == 0) continue;
        int const low = 31 - __clz(nib);
        int const d = column_top(e.board[col0 + i] & ~((2u << low) - 1u)) - low - 1;
        drop = d < drop ? d : drop;
    }
    uint32_t full = FIELD;
    for (int i = 0; i < 4; ++i) {
        uint32_t const nib = (cols >> (4 * i)) & 0xFu;
        if (nib) e.board[col0 + i] |= nib << drop;
    }
    for (int c = 0; c < W; ++c) full &= e.board[c];
    int const cleared = __popc(full);
    if (full)
        for (int c = 0; c < W; ++c) e.board[c] = clear_rows(e.board[c], full);
    advance_queue(e);
    update_game_over(e);
    return e.over ? -1 : cleared;
}

// ------------------------------------------------------------ value model ---
// Integer board metrics of ta3_ai/incl/ta3/ai/models/metrics/v_board_metrics.hpp:130-225.
struct BoardInts {
    uint32_t holes, hole_depths, max_height, wells;
    int surf_sq;
};

__device__ __forceinline__ BoardInts board_ints(uint32_t const (&b)[W]) {
    BoardInts r{0, 0, 0, 0, 0};
    int h[W];
#pragma unroll
    for (int x = 0; x < W; ++x) {
        uint32_t const col = b[x];
        h[x] = H - column_top(col);
        int const n = __popc(col);
        r.holes += uint32_t(h[x] - n);
        r.max_height = max(r.max_height, uint32_t(h[x]));
        // sum of occupied row indices via the 5 bit planes of the row index
        int const s = __popc(col & 0x2AAAAAu) + 2 * __popc(col & 0x4CCCCCu) + 4 * __popc(col & 0x70F0F0u) +
                      8 * __popc(col & 0x00FF00u) + 16 * __popc(col & 0x7F0000u);
        // (H-1)n + n(n+1)/2 - (s + n^2): occupied cells' count of empty cells beneath them
        r.hole_depths += uint32_t((H - 1) * n + n * (n + 1) / 2 - (s + n * n));
    }
#pragma unroll
    for (int x = 1; x < W; ++x) {
        int const d = h[x] - h[x - 1];
        r.surf_sq += d * d;
    }
    uint32_t wells = (h[1] >= h[0] + 3) + (h[W - 2] >= h[W - 1] + 3);
#pragma unroll
    for (int x = 1; x < W - 1; ++x) wells += (h[x - 1] >= h[x] + 3 && h[x + 1] >= h[x] + 3);
    r.wells = wells;
    return r;
}

struct Model {                       // 97 v11 weights, model_v11.hpp:166-180 layout
    float w[NPARAMS];
};

// ModelV11::extractInputs + forward (model_v11.hpp:63-91,166-180; utility.hpp:30-46),
// each multiply and add rounded separately in the reference order.
__device__ __forceinline__ float evaluate(uint32_t clear_bits, uint32_t const (&b)[W], bool held_i, Model const& m) {
    BoardInts const bi = board_ints(b);
    float in[NIN];
#pragma unroll
    for (int k = 0; k < 4; ++k) in[k] = __fmul_rn(float((clear_bits >> (8 * k)) & 0xFFu), 0.25f);
    float const sv = bi.surf_sq > 0 ? __fsqrt_rn(float(bi.surf_sq)) : 0.0f;
    in[4] = __fdiv_rn(sv, 100.0f);
    in[5] = __fdiv_rn(float(bi.holes), 20.0f);
    in[6] = __fdiv_rn(float(bi.hole_depths), 200.0f);
    in[7] = float(bi.max_height);
    in[8] = held_i ? 1.0f : 0.0f;
    in[9] = __fdiv_rn(float(bi.wells), 5.0f);
    float hid[NHID];
#pragma unroll
    for (int o = 0; o < NHID; ++o) {
        float v = m.w[NIN * NHID + o];
#pragma unroll
        for (int i = 0; i < NIN; ++i) v = __fadd_rn(v, __fmul_rn(in[i], m.w[o * NIN + i]));
        hid[o] = v > 0.0f ? v : 0.0f;
    }
    float v = m.w[NIN * NHID + NHID + NHID];
#pragma unroll
    for (int i = 0; i < NHID; ++i) v = __fadd_rn(v, __fmul_rn(hid[i], m.w[NIN * NHID + NHID + i]));
    return v;
}

// ------------------------------------------------------------- candidate ---
// search.hpp:61-70 apply(): spawn-collision + drop (board2.hpp:306-320), lock
// (board2.hpp:322-327) and line clear (board2.hpp:333-342). Returns legality;
// nb receives the resulting board and cleared the rows removed.
__device__ __forceinline__ bool apply(uint32_t const (&b)[W], uint32_t pl, uint32_t (&nb)[W], int& cleared) {
    uint32_t const cols = pl & 0xFFFFu;
    int const col0 = int((pl >> 16) & 0xFu);
    uint32_t hit = 0;
    int drop = H;
    uint32_t nib[W];
#pragma unroll
    for (int x = 0; x < W; ++x) {
        uint32_t const d = uint32_t(x - col0);
        nib[x] = d < 4u ? (cols >> (4u * d)) & 0xFu : 0u;
        hit |= b[x] & nib[x];
        int const low = 31 - __clz(nib[x] | 1u);
        int const dd = column_top(b[x] & ~((2u << low) - 1u)) - low - 1;
        drop = (nib[x] != 0u && dd < drop) ? dd : drop;
    }
    if (hit) return false;
    uint32_t full = FIELD;
#pragma unroll
    for (int x = 0; x < W; ++x) {
        nb[x] = b[x] | (nib[x] << drop);
        full &= nb[x];
    }
    cleared = __popc(full);
    if (full) {
#pragma unroll
        for (int x = 0; x < W; ++x) nb[x] = clear_rows(nb[x], full);
    }
    return true;
}

__device__ __forceinline__ void load_board(uint32_t const* __restrict__ src, uint32_t (&b)[W]) {
    uint4 const q0 = *reinterpret_cast<uint4 const*>(src);
    uint4 const q1 = *reinterpret_cast<uint4 const*>(src + 4);
    uint2 const q2 = *reinterpret_cast<uint2 const*>(src + 8);
    b[0] = q0.x; b[1] = q0.y; b[2] = q0.z; b[3] = q0.w;
    b[4] = q1.x; b[5] = q1.y; b[6] = q1.z; b[7] = q1.w;
    b[8] = q2.x; b[9] = q2.y;
}

// ------------------------------------------------------------------ top-K ---
__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    return (uint64_t(__shfl_sync(0xFFFFFFFFu, uint32_t(v >> 32), src)) << 32) |
           __shfl_sync(0xFFFFFFFFu, uint32_t(v), src);
}
__device__ __forceinline__ uint64_t shfl64_up(uint64_t v) {
    return (uint64_t(__shfl_up_sync(0xFFFFFFFFu, uint32_t(v >> 32), 1)) << 32) |
           __shfl_up_sync(0xFFFFFFFFu, uint32_t(v), 1);
}

// Fold one key per lane into the warp's sorted top-K list (lane i = i-th
// largest, 0 = empty). Keys are unique per level (the low word encodes the
// slot), so the kept set equals beam.hpp:244-265's "max score, lowest slot on
// ties" whatever the insertion order.
__device__ __forceinline__ void topk_fold(uint64_t& list, uint64_t key, int k, int lane) {
    uint64_t thr = shfl64(list, k - 1);
    uint32_t mask = __ballot_sync(0xFFFFFFFFu, key > thr);
    while (mask) {
        int const s = __ffs(int(mask)) - 1;
        uint64_t const x = shfl64(key, s);
        int const pos = __popc(__ballot_sync(0xFFFFFFFFu, list > x));
        uint64_t const up = shfl64_up(list);
        if (lane > pos && lane < k) list = up;
        if (lane == pos) list = x;
        thr = shfl64(list, k - 1);
        mask &= ~(1u << s);
        mask &= __ballot_sync(0xFFFFFFFFu, key > thr);
    }
}

__device__ __forceinline__ uint64_t warp_max64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t const u = shfl64(v, (threadIdx.x + o) & 31);
        v = u > v ? u : v;
    }
    return v;
}

// ---------------------------------------------------------------- kernel ---
struct alignas(16) WarpShared {
    uint32_t fboard[32][12];          // kept frontier boards (rank -> board), 48-byte rows
    Engine eng;                        // the committed game
    uint32_t seg_off[65];              // per-level candidate segments (parent, child list)
    uint32_t seg_info[64];
    Stats st;
};

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
    uint32_t* scratch;                 // [0] sim ticket, [1] error status
    uint32_t num_games, models_per_island, max_moves, total_sims;
};

struct Move {
    int orient, x, hold;
    bool none;
};

// Build one level's segment table: segment j = (parent rank j/2, child j%2);
// each spans the child piece's placement count. Returns the candidate total.
__device__ __forceinline__ uint32_t build_segments(WarpShared& ws, uint32_t const* slot_piece, int tree, int level,
                                                   uint32_t fnode, int kept, int lane) {
    uint32_t base = 0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        int const j = lane + 32 * half;
        int const k = j >> 1;
        uint32_t const pnode = __shfl_sync(0xFFFFFFFFu, fnode, k & 31);
        uint32_t const cnode = 2u * pnode + uint32_t(j & 1);
        uint32_t const info = c_tables.node[tree][level][cnode & 15u];
        uint32_t const piece = slot_piece[info & 0xFu];
        uint32_t const held_slot = (info >> 4) & 0xFu;
        uint32_t const held_i = held_slot != HELD_NONE && slot_piece[held_slot] == 0u;
        uint32_t const cnt = k < kept ? c_tables.nplace[piece] : 0u;
        // inclusive warp scan of cnt
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t const n = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += n;
        }
        ws.seg_off[j] = base + incl - cnt;
        ws.seg_info[j] = uint32_t(k) | (piece << 8) | (held_i << 12) | (cnode << 16);
        base += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) ws.seg_off[64] = base;
    __syncwarp();
    return base;
}

__device__ __forceinline__ Move search_move(WarpShared& ws, Model const& m, int lane, uint32_t& evals, uint32_t* status) {
    Move mv{0, 0, 0, true};
    if (ws.eng.over) return mv;
    uint32_t slot_piece[NSLOTS];                                  // beam.hpp:226-237
    slot_piece[0] = ws.eng.held;
    slot_piece[1] = ws.eng.queue[0];
#pragma unroll
    for (int i = 0; i < DEPTH; ++i) slot_piece[2 + i] = ws.eng.queue[1 + i];
    int const tree = ws.eng.held == NO_PIECE ? 1 : 0;

    // ---- root stage: score every legal root, keep the best K0 (beam.hpp:283-301,507-513)
    uint32_t const r0 = c_tables.node[tree][0][0], r1 = c_tables.node[tree][0][1];
    uint32_t const p0 = slot_piece[r0 & 0xFu], p1 = slot_piece[r1 & 0xFu];
    uint32_t const h0 = (r0 >> 4) & 0xFu, h1 = (r1 >> 4) & 0xFu;
    bool const hi0 = h0 != HELD_NONE && slot_piece[h0] == 0u;
    bool const hi1 = h1 != HELD_NONE && slot_piece[h1] == 0u;
    uint32_t const n0 = c_tables.nplace[p0], ntot = n0 + c_tables.nplace[p1];
    uint32_t root_board[W];
    load_board(ws.eng.board, root_board);
    uint64_t list = 0;
    for (uint32_t c0 = 0; c0 < ntot; c0 += WARP) {
        uint32_t const c = c0 + uint32_t(lane);
        uint64_t key = 0;
        if (c < ntot) {
            bool const g = c >= n0;
            uint32_t const i = g ? c - n0 : c;
            uint32_t const pl = c_tables.place[g ? p1 : p0][i];
            uint32_t nb[W];
            int cl;
            if (apply(root_board, pl, nb, cl)) {
                ++evals;
                float const v = evaluate(clear_bump(cl), nb, g ? hi1 : hi0, m);
                uint32_t const slot = (g ? MP : 0u) + i;
                key = (uint64_t(ordered_bits(v)) << 32) | uint64_t(0xFFFFFFFFu - slot);
            }
        }
        topk_fold(list, key, K0, lane);
    }
    int kept = __popc(__ballot_sync(0xFFFFFFFFu, list != 0));
    if (kept == 0) return mv;                                     // no legal root: game over

    // ---- seed the frontier (beam.hpp:307-329): lane k = rank k
    uint32_t const root_slot = 0xFFFFFFFFu - uint32_t(list);      // lanes < kept
    uint32_t fclears = 0, fscore = uint32_t(list >> 32), fnode = 0, frank = uint32_t(lane);
    if (lane < kept) {
        uint32_t const g = root_slot / MP;
        uint32_t const pl = c_tables.place[g ? p1 : p0][root_slot % MP];
        uint32_t nb[W];
        int cl = 0;
        apply(root_board, pl, nb, cl);
        fclears = clear_bump(cl);
        fnode = g;
#pragma unroll
        for (int x = 0; x < W; ++x) ws.fboard[lane][x] = nb[x];
    }
    __syncwarp();

    uint64_t best = 0;                                            // leaf-order (score | order) maximum
    // ---- middle levels (beam.hpp:540-564)
#pragma unroll 1
    for (int level = 1; level + 1 < DEPTH; ++level) {
        int const kl = level == 1 ? K1 : K2;
        uint32_t const total = build_segments(ws, slot_piece, tree, level, fnode, kept, lane);
        uint64_t klist = 0;
        uint32_t has_child = 0;
        int seg = 0;
        for (uint32_t c0 = 0; c0 < total; c0 += WARP) {
            uint32_t const c = c0 + uint32_t(lane);
            uint64_t key = 0;
            uint32_t info = 0, i = 0;
            if (c < total) {
                while (ws.seg_off[seg + 1] <= c) ++seg;
                info = ws.seg_info[seg];
                i = c - ws.seg_off[seg];
            }
            uint32_t const k = info & 0xFFu;
            uint32_t const pclears = __shfl_sync(0xFFFFFFFFu, fclears, int(k));
            if (c < total) {
                uint32_t b[W];
                load_board(ws.fboard[k], b);
                uint32_t const pl = c_tables.place[(info >> 8) & 0xFu][i];
                uint32_t nb[W];
                int cl;
                if (apply(b, pl, nb, cl)) {
                    ++evals;
                    has_child |= 1u << k;
                    float const v = evaluate(pclears + clear_bump(cl), nb, (info >> 12) & 1u, m);
                    uint32_t const slot = (k * 2u + (uint32_t(seg) & 1u)) * MP + i;
                    key = (uint64_t(ordered_bits(v)) << 32) | uint64_t(0xFFFFFFFFu - slot);
                }
            }
            topk_fold(klist, key, kl, lane);
        }
        has_child = __reduce_or_sync(0xFFFFFFFFu, has_child);
        // kept nodes with no legal continuation become leaves at this depth (beam.hpp:549-551)
        if (lane < kept && !((has_child >> lane) & 1u)) {
            uint64_t const fk = (uint64_t(fscore) << 32) | uint64_t(ORDER_SPAN - (LEAF_ORDERS + frank));
            best = fk > best ? fk : best;
        }
        int const next = __popc(__ballot_sync(0xFFFFFFFFu, klist != 0));
        // advance the frontier (beam.hpp:379-403): lane j builds kept node j
        uint32_t const sslot = 0xFFFFFFFFu - uint32_t(klist);
        uint32_t const pk = next > lane ? sslot / (2 * MP) : 0u;
        uint32_t const child = (sslot / MP) & 1u;
        uint32_t const par_clears = __shfl_sync(0xFFFFFFFFu, fclears, int(pk));
        uint32_t const par_node = __shfl_sync(0xFFFFFFFFu, fnode, int(pk));
        uint32_t const par_rank = __shfl_sync(0xFFFFFFFFu, frank, int(pk));
        uint32_t nb[W];
        uint32_t ncl = 0, nnode = 0;
        if (lane < next) {
            uint32_t const cnode = 2u * par_node + child;
            uint32_t const piece = slot_piece[c_tables.node[tree][level][cnode] & 0xFu];
            uint32_t b[W];
            load_board(ws.fboard[pk], b);
            int cl = 0;
            apply(b, c_tables.place[piece][sslot % MP], nb, cl);
            ncl = par_clears + clear_bump(cl);
            nnode = cnode;
        }
        __syncwarp();
        if (lane < next) {
#pragma unroll
            for (int x = 0; x < W; ++x) ws.fboard[lane][x] = nb[x];
        }
        __syncwarp();
        fclears = ncl;
        fscore = uint32_t(klist >> 32);
        fnode = nnode;
        frank = par_rank;
        kept = next;
    }

    // ---- leaf stage (beam.hpp:407-443): argmax over leaves and per-list fallbacks
    {
        uint32_t const total = build_segments(ws, slot_piece, tree, DEPTH - 1, fnode, kept, lane);
        uint32_t legal_lo = 0, legal_hi = 0;
        int seg = 0;
        for (uint32_t c0 = 0; c0 < total; c0 += WARP) {
            uint32_t const c = c0 + uint32_t(lane);
            uint32_t info = 0, i = 0;
            if (c < total) {
                while (ws.seg_off[seg + 1] <= c) ++seg;
                info = ws.seg_info[seg];
                i = c - ws.seg_off[seg];
            }
            uint32_t const k = info & 0xFFu;
            uint32_t const pclears = __shfl_sync(0xFFFFFFFFu, fclears, int(k));
            if (c < total) {
                uint32_t b[W];
                load_board(ws.fboard[k], b);
                uint32_t const pl = c_tables.place[(info >> 8) & 0xFu][i];
                uint32_t nb[W];
                int cl;
                if (apply(b, pl, nb, cl)) {
                    ++evals;
                    if (seg < 32) legal_lo |= 1u << seg;
                    else legal_hi |= 1u << (seg - 32);
                    float const v = evaluate(pclears + clear_bump(cl), nb, (info >> 12) & 1u, m);
                    uint32_t const order = (k * 2u + (uint32_t(seg) & 1u)) * MP + i;
                    uint64_t const key = (uint64_t(ordered_bits(v)) << 32) | uint64_t(ORDER_SPAN - order);
                    best = key > best ? key : best;
                }
            }
        }
        legal_lo = __reduce_or_sync(0xFFFFFFFFu, legal_lo);
        legal_hi = __reduce_or_sync(0xFFFFFFFFu, legal_hi);
        // a list whose piece never fit: the frontier board is the leaf (beam.hpp:439-440)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            int const j = lane + 32 * half;
            int const k = j >> 1;
            uint32_t const sc = __shfl_sync(0xFFFFFFFFu, fscore, k & 31);
            bool const legal = ((half ? legal_hi : legal_lo) >> lane) & 1u;
            if (k < kept && !legal) {
                uint64_t const key = (uint64_t(sc) << 32) | uint64_t(ORDER_SPAN - uint32_t(j) * MP);
                best = key > best ? key : best;
            }
        }
    }
    best = warp_max64(best);
    if (best == 0) {                                              // unreachable with >= 1 root
        if (lane == 0) atomicOr(status, 1u);
        return mv;
    }
    // ---- decode the winning key back to its root move (beam.hpp:450-470)
    uint32_t const order = ORDER_SPAN - uint32_t(best);
    uint32_t const leaf_rank = __shfl_sync(0xFFFFFFFFu, frank, int((order / (2 * MP)) & 31u));
    uint32_t const rank = order >= uint32_t(LEAF_ORDERS) ? order - LEAF_ORDERS : leaf_rank;
    uint32_t const rs = __shfl_sync(0xFFFFFFFFu, root_slot, int(rank & 31u));
    uint32_t const g = rs / MP;
    uint32_t const pl = c_tables.place[g ? p1 : p0][rs % MP];
    mv.orient = int((pl >> 20) & 3u);
    mv.x = int((pl >> 24) & 0xFu) - 2;
    mv.hold = int((c_tables.node[tree][0][g] >> 8) & 1u);
    mv.none = ordered_bits_inv(uint32_t(best >> 32)) == -__int_as_float(0x7f800000);   // search.hpp:41
    return mv;
}

// stats_v4::advance (tetris_stats.hpp:19-23 with metrics.hpp:196-229)
__device__ void stats_advance(Stats& st, uint32_t const* board, uint32_t lines) {
    uint32_t b[W];
    for (int x = 0; x < W; ++x) b[x] = board[x];
    BoardInts const bi = board_ints(b);
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

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) eval_kernel(Params p) {
    __shared__ WarpShared s_warp[WARPS];
    int const lane = int(threadIdx.x & 31u);
    WarpShared& ws = s_warp[threadIdx.x >> 5];
    for (;;) {
        uint32_t sim = 0;
        if (lane == 0) sim = atomicAdd(&p.scratch[0], 1u);
        sim = __shfl_sync(0xFFFFFFFFu, sim, 0);
        if (sim >= p.total_sims) break;
        uint32_t const mdl = sim / p.num_games, g = sim % p.num_games;
        uint32_t const island = mdl / p.models_per_island;
        uint64_t const seed = p.seeds[size_t(island) * p.num_games + g];
        Model m;
        float const* wsrc = p.weights + size_t(mdl) * NPARAMS;
#pragma unroll
        for (int i = 0; i < NPARAMS; ++i) m.w[i] = __ldg(wsrc + i);
        if (lane == 0) {
            engine_reset(ws.eng, seed);
            ws.st = Stats{};
        }
        __syncwarp();
        uint32_t evals = 0, moves = 0;
        for (uint32_t mv_i = 0; mv_i < p.max_moves && !ws.eng.over; ++mv_i) {   // model_eval_host.cpp:39-50
            Move const mv = search_move(ws, m, lane, evals, &p.scratch[1]);
            if (mv.none) break;
            if (lane == 0) {
                if (p.trace) {
                    uint8_t* t = p.trace + (size_t(sim) * p.max_moves + moves) * 3;
                    t[0] = uint8_t(mv.hold);
                    t[1] = uint8_t(mv.orient);
                    t[2] = uint8_t(mv.x + 2);
                }
                if (mv.hold) engine_hold(ws.eng);
                int const cl = engine_place(ws.eng, mv.orient, mv.x);
                if (cl >= 0) stats_advance(ws.st, ws.eng.board, uint32_t(cl));
                else ws.eng.over = 2;                                // DIED: stop without a stats update
            }
            ++moves;
            __syncwarp();
            if (ws.eng.over == 2) break;
        }
        evals = __reduce_add_sync(0xFFFFFFFFu, evals);
        if (lane == 0) {
            p.score[sim] = final_score(ws.st);
            if (p.pieces) p.pieces[sim] = ws.st.pieces;
            if (p.lines) p.lines[sim] = ws.st.lines;
            if (p.evals) p.evals[sim] = evals;
            if (p.n_moves) p.n_moves[sim] = moves;
            if (p.board_out)
                for (int x = 0; x < W; ++x) p.board_out[size_t(sim) * W + x] = ws.eng.board[x];
        }
        __syncwarp();
    }
}

constexpr int kWarpsPerBlock = 4;

} // namespace
} // namespace ta3b

// ===================================================================== C ABI ===
using namespace ta3b;

struct ta3b_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t warps_per_block = kWarpsPerBlock;
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

int check_sizes(ta3b_ctx* ctx, uint32_t num_islands, uint32_t models_per_island, uint32_t num_params,
                uint32_t num_games) {
    if (!ctx) return fail(ctx, TA3B_ERR_ARG, "null context");
    if (num_params != NPARAMS)
        return fail(ctx, TA3B_ERR_ARG, "num_params must be " + std::to_string(NPARAMS) + " (v11 value model)");
    uint64_t const sims = uint64_t(num_islands) * models_per_island * num_games;
    if (sims > 0xFFFFFFF0ull) return fail(ctx, TA3B_ERR_ARG, "too many sims in one batch");
    return TA3B_OK;
}

int launch(ta3b_ctx* ctx, Params const& prm, cudaStream_t st) {
    if (prm.total_sims == 0) return TA3B_OK;
    TA3B_CUDA(ctx, cudaMemsetAsync(prm.scratch, 0, 2 * sizeof(uint32_t), st), "reset work queue");
    uint32_t const need_blocks = (prm.total_sims + ctx->warps_per_block - 1) / ctx->warps_per_block;
    uint32_t const grid = need_blocks < ctx->grid ? need_blocks : ctx->grid;
    eval_kernel<kWarpsPerBlock><<<grid, ctx->warps_per_block * 32, 0, st>>>(prm);
    TA3B_CUDA(ctx, cudaGetLastError(), "kernel launch");
    return TA3B_OK;
}

int read_status(ta3b_ctx* ctx) {
    uint32_t status = 0;
    TA3B_CUDA(ctx, cudaMemcpyAsync(&status, ctx->d_scratch + 1, sizeof status, cudaMemcpyDeviceToHost, ctx->stream),
              "read status");
    TA3B_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "kernel run");
    if (status) return fail(ctx, TA3B_ERR_DEVICE, "kernel reported status " + std::to_string(status));
    return TA3B_OK;
}

int host_eval(ta3b_ctx* ctx, float const* weights, uint32_t num_islands, uint32_t mpi, uint32_t num_params,
              uint64_t const* seeds, uint32_t num_games, uint32_t max_moves, float* score_out, uint32_t* pieces_out,
              uint32_t* lines_out, uint32_t* evals_out, uint8_t* trace_out, uint32_t* nmoves_out,
              uint32_t* board_out) {
    if (int rc = check_sizes(ctx, num_islands, mpi, num_params, num_games)) return rc;
    uint64_t const models = uint64_t(num_islands) * mpi;
    uint64_t const sims = models * num_games;
    if (sims == 0) return TA3B_OK;
    if (!weights || !seeds || !score_out) return fail(ctx, TA3B_ERR_ARG, "null weights / seeds / score_out");
    TA3B_CUDA(ctx, cudaSetDevice(ctx->device), "set device");
    if (int rc = grow(ctx, ctx->d_w, ctx->cap_w, models * NPARAMS, "alloc weights")) return rc;
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
    bool const tracing = trace_out || nmoves_out || board_out;
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
    TA3B_CUDA(ctx, cudaMemcpyAsync(ctx->d_w, weights, models * NPARAMS * sizeof(float), cudaMemcpyHostToDevice,
                                   ctx->stream), "copy weights");
    TA3B_CUDA(ctx, cudaMemcpyAsync(ctx->d_seeds, seeds, uint64_t(num_islands) * num_games * sizeof(uint64_t),
                                   cudaMemcpyHostToDevice, ctx->stream), "copy seeds");
    Params prm{};
    prm.weights = ctx->d_w;
    prm.seeds = ctx->d_seeds;
    prm.score = ctx->d_score;
    prm.pieces = ctx->d_pieces;
    prm.lines = ctx->d_lines;
    prm.evals = ctx->d_evals;
    prm.trace = tracing ? ctx->d_trace : nullptr;
    prm.n_moves = tracing ? ctx->d_nmoves : nullptr;
    prm.board_out = tracing ? ctx->d_board : nullptr;
    prm.scratch = ctx->d_scratch;
    prm.num_games = num_games;
    prm.models_per_island = mpi;
    prm.max_moves = max_moves;
    prm.total_sims = uint32_t(sims);
    if (int rc = launch(ctx, prm, ctx->stream)) return rc;
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
    return read_status(ctx);
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
    if (c.warps_per_block && c.warps_per_block != kWarpsPerBlock) {
        g_create_error = "warps_per_block must be 0 or " + std::to_string(kWarpsPerBlock);
        delete ctx;
        return nullptr;
    }
    if (cudaSetDevice(c.device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_scratch, 4 * sizeof(uint32_t)) != cudaSuccess) {
        g_create_error = std::string("context setup: ") + cudaGetErrorString(cudaGetLastError());
        ta3b_destroy(ctx);
        return nullptr;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eval_kernel<kWarpsPerBlock>, kWarpsPerBlock * 32, 0);
    if (per_sm < 1) per_sm = 1;
    ctx->blocks_per_sm = c.blocks_per_sm ? (c.blocks_per_sm < uint32_t(per_sm) ? c.blocks_per_sm : uint32_t(per_sm))
                                         : uint32_t(per_sm);
    ctx->grid = ctx->sms * ctx->blocks_per_sm;
    return ctx;
}

void ta3b_destroy(ta3b_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    void* bufs[] = {ctx->d_w, ctx->d_seeds, ctx->d_score, ctx->d_pieces, ctx->d_lines, ctx->d_evals,
                    ctx->d_trace, ctx->d_nmoves, ctx->d_board, ctx->d_scratch};
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
                    uint32_t* n_moves_out, uint32_t* board_out) {
    return host_eval(ctx, weights, 1, num_models, num_params, seeds, num_games, max_moves, score_out, pieces_out,
                     lines_out, evals_out, trace_out, n_moves_out, board_out);
}

int ta3b_eval_device(ta3b_ctx* ctx, float const* d_weights, uint32_t num_islands, uint32_t models_per_island,
                     uint32_t num_params, uint64_t const* d_seeds, uint32_t num_games, uint32_t max_moves,
                     float* d_score, uint32_t* d_pieces, uint32_t* d_lines, uint32_t* d_evals, void* stream) {
    if (int rc = check_sizes(ctx, num_islands, models_per_island, num_params, num_games)) return rc;
    uint64_t const sims = uint64_t(num_islands) * models_per_island * num_games;
    if (sims == 0) return TA3B_OK;
    if (!d_weights || !d_seeds || !d_score) return fail(ctx, TA3B_ERR_ARG, "null device pointer");
    Params prm{};
    prm.weights = d_weights;
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
    return launch(ctx, prm, stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
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

int ta3b_launch_info(ta3b_ctx const* ctx, uint32_t* grid, uint32_t* warps_per_block, uint32_t* sms) {
    if (!ctx) return TA3B_ERR_ARG;
    if (grid) *grid = ctx->grid;
    if (warps_per_block) *warps_per_block = ctx->warps_per_block;
    if (sms) *sms = ctx->sms;
    return TA3B_OK;
}

} // extern "C"
