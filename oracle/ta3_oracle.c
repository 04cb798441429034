/*
 * ta3_oracle.c -- CPU restatement of the reference's model x game beam-search
 * evaluation (codethinki/tetris_ai3: ta3_sim + ta3_ai + ta3_gpu eval_host).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity oracle: tests/, the
 * smoke() check in __graft_entry__.py and the cpu_baseline leg of bench.py may
 * load it (as oracle/_build/libta3oracle.so) to CHECK the CUDA path. The
 * product (tetris_ai3_b200) never links, loads or calls it, and has no CPU
 * fallback.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against golden vectors generated by running the reference's own CPU code
 * (oracle/_ref, built by oracle/Makefile from the reference sources) and
 * against the reference tests' known-answer facts.
 *
 * Every function names the reference file:line it restates. Floating point
 * follows the reference CPU path exactly: FP32 value model with separate
 * multiply / add roundings in the reference order (compile with
 * -ffp-contract=off), IEEE sqrtf and division, FP64 final score.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <string.h>

#define W 10          /* ta3_sim/incl/ta3/sim/utility/tetris_defs.hpp:9 (COLS)  */
#define H 23          /* ta3_sim/incl/ta3/sim/utility/tetris_defs.hpp:9 (ROWS)  */
#define FIELD ((1u << H) - 1u)  /* board2.hpp:154 */
#define FLOOR (1u << H)         /* board2.hpp:157 */
#define NPIECE 7
#define NO_PIECE 7              /* piece_defs.hpp:31 */
#define QUEUE 6                 /* tetris_defs.hpp:12 */
#define DEPTH 4                 /* variation_sequences.hpp:22,25: widths {16,32,32} */
#define MP 34                   /* placements.hpp:223 */
#define NSLOTS (DEPTH + 2)      /* variation_sequences.hpp:51 */
#define HELD_NONE 7             /* variation_sequences.hpp:137 */
#define NPARAMS 97              /* model_v11.hpp:44 */
#define NIN 10
#define NHID 8

static const uint32_t KS[DEPTH - 1] = {16, 32, 32};   /* variation_sequences.hpp:22 */

/* ---------------------------------------------------------------- bits --- */
static int ctz32(uint32_t v) { return v ? __builtin_ctz(v) : 32; }
static int popc32(uint32_t v) { return __builtin_popcount(v); }
static int bitw32(uint32_t v) { return v ? 32 - __builtin_clz(v) : 0; }

/* ----------------------------------------- xoshiro256ss.hpp:12-61 --- */
typedef struct { uint64_t s[4]; } rng_t;

static void rng_seed(rng_t* r, uint64_t s) {           /* xoshiro256ss.hpp:20-28 */
    for (int i = 0; i < 4; ++i) {
        s += 0x9e3779b97f4a7c15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        r->s[i] = z ^ (z >> 31);
    }
}
static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t* r) {                    /* xoshiro256ss.hpp:33-45 */
    uint64_t const res = rotl64(r->s[1] * 5, 7) * 9;
    uint64_t const t = r->s[1] << 17;
    r->s[2] ^= r->s[0];
    r->s[3] ^= r->s[1];
    r->s[1] ^= r->s[2];
    r->s[0] ^= r->s[3];
    r->s[2] ^= t;
    r->s[3] = rotl64(r->s[3], 45);
    return res;
}

/* --------------------------------- piece geometry, piece_offsets.hpp --- */
/* Block coordinates per (piece, orientation), piece_offsets.hpp:19-85.
 * Piece order I,O,T,S,Z,J,L (piece_defs.hpp:19-29); orientation order
 * TOP,RIGHT,BOTTOM,LEFT (piece_defs.hpp:129-136). */
static const int8_t BLOCKS[NPIECE][4][4][2] = {
    /* I */ {{{0,1},{1,1},{2,1},{3,1}}, {{2,0},{2,1},{2,2},{2,3}}, {{0,2},{1,2},{2,2},{3,2}}, {{1,0},{1,1},{1,2},{1,3}}},
    /* O */ {{{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}},
    /* T */ {{{1,0},{0,1},{1,1},{2,1}}, {{1,0},{1,1},{2,1},{1,2}}, {{0,1},{1,1},{2,1},{1,2}}, {{1,0},{0,1},{1,1},{1,2}}},
    /* S */ {{{1,0},{2,0},{0,1},{1,1}}, {{0,0},{0,1},{1,1},{1,2}}, {{1,1},{2,1},{1,2},{0,2}}, {{1,0},{1,1},{2,1},{2,2}}},
    /* Z */ {{{0,0},{1,0},{1,1},{2,1}}, {{2,0},{1,1},{2,1},{1,2}}, {{1,1},{0,1},{1,2},{2,2}}, {{1,0},{0,1},{1,1},{0,2}}},
    /* J */ {{{0,0},{0,1},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{1,2}}, {{0,1},{1,1},{2,1},{2,2}}, {{1,0},{1,1},{0,2},{1,2}}},
    /* L */ {{{2,0},{0,1},{1,1},{2,1}}, {{1,0},{1,1},{1,2},{2,2}}, {{0,1},{1,1},{2,1},{0,2}}, {{0,0},{1,0},{1,1},{1,2}}},
};

typedef struct { uint16_t cols; int8_t left; uint8_t ncols; } oshape_t;
static oshape_t SHAPES[NPIECE][4];                       /* piece_offsets.hpp:186-201 */

typedef struct { uint8_t orient; int8_t x; uint16_t cols; int8_t col0; } placement_t;
static placement_t PLACEMENTS[NPIECE][MP];               /* placements.hpp:189-205 */
static uint32_t NPLACE[NPIECE];                          /* placements.hpp:210-212 */

/* plan tree, beam.hpp:49-128; node tuple per layer */
typedef struct { uint8_t slot, parent, cbeg, cend, root_hold, held_slot; } node_t;
typedef struct { node_t nodes[DEPTH][1u << DEPTH]; uint8_t count[DEPTH]; } tree_t;
static tree_t TREES[2];

static int g_ready = 0;

static void build_shapes(void) {
    for (int t = 0; t < NPIECE; ++t)
        for (int o = 0; o < 4; ++o) {
            uint32_t box[4] = {0, 0, 0, 0};                  /* piece_offsets.hpp:112-119 */
            for (int b = 0; b < 4; ++b)
                box[BLOCKS[t][o][b][0]] |= 1u << BLOCKS[t][o][b][1];
            int left = 0;                                   /* piece_offsets.hpp:132-143 */
            while (left < 4 && box[left] == 0) ++left;
            int right = 4;
            while (right > left && box[right - 1] == 0) --right;
            uint16_t cols = 0;
            for (int c = 0; c < right - left; ++c) cols |= (uint16_t)(box[left + c] << (4 * c));
            SHAPES[t][o].cols = cols;
            SHAPES[t][o].left = (int8_t)left;
            SHAPES[t][o].ncols = (uint8_t)(right - left);
        }
}

/* placements.hpp:107-125: vertically normalised occupied-column signature */
static void signature(int t, int o, uint32_t sig[4], uint32_t* n) {
    oshape_t const s = SHAPES[t][o];
    uint32_t minbit = 32;
    for (int c = 0; c < s.ncols; ++c) {
        uint32_t const v = (s.cols >> (4 * c)) & 0xFu;
        if (v) { uint32_t const b = (uint32_t)ctz32(v); if (b < minbit) minbit = b; }
    }
    if (minbit == 32) minbit = 0;
    *n = s.ncols;
    for (int c = 0; c < 4; ++c) sig[c] = c < s.ncols ? (((s.cols >> (4 * c)) & 0xFu) >> minbit) : 0;
}

static void build_placements(void) {                    /* placements.hpp:142-205 */
    for (int t = 0; t < NPIECE; ++t) {
        uint32_t seen[4][4]; uint32_t seenN[4]; int nseen = 0; uint32_t w = 0;
        for (int o = 0; o < 4; ++o) {
            uint32_t sig[4], n;
            signature(t, o, sig, &n);
            int dup = 0;
            for (int j = 0; j < nseen && !dup; ++j)
                if (seenN[j] == n && memcmp(seen[j], sig, sizeof sig) == 0) dup = 1;
            if (dup) continue;
            memcpy(seen[nseen], sig, sizeof sig); seenN[nseen] = n; ++nseen;
            int const xmin = -SHAPES[t][o].left;           /* placements.hpp:70-75 */
            int const xmax = W - SHAPES[t][o].left - SHAPES[t][o].ncols;
            for (int x = xmin; x <= xmax; ++x) {
                PLACEMENTS[t][w].orient = (uint8_t)o;
                PLACEMENTS[t][w].x = (int8_t)x;
                PLACEMENTS[t][w].cols = SHAPES[t][o].cols;
                PLACEMENTS[t][w].col0 = (int8_t)(x + SHAPES[t][o].left);   /* piece_offsets.hpp:206-209 */
                ++w;
            }
        }
        NPLACE[t] = w;
    }
}

/* variation_sequences.hpp:216-255 (build_plans) + beam.hpp:69-126 (build_tree) */
static void build_trees(void) {
    for (int he = 0; he < 2; ++he) {
        int const held_empty = he == 1;
        uint8_t pslot[1u << DEPTH][DEPTH], pheld[1u << DEPTH][DEPTH], proot[1u << DEPTH];
        for (uint32_t d = 0; d < (1u << DEPTH); ++d) {
            uint8_t cur = 1, hld = 0; int empty = held_empty; uint32_t k = 1;
            for (uint32_t i = 0; i < DEPTH; ++i) {
                int did = 0;
                if (d & (1u << i)) {
                    if (empty) { hld = cur; cur = (uint8_t)(1 + k++); empty = 0; }
                    else { uint8_t const tmp = cur; cur = hld; hld = tmp; }
                    did = 1;
                }
                pslot[d][i] = cur;
                if (i == 0) proot[d] = (uint8_t)did;
                pheld[d][i] = empty ? HELD_NONE : hld;
                if (i + 1 < DEPTH) cur = (uint8_t)(1 + k++);
            }
        }
        tree_t* tr = &TREES[he];
        memset(tr, 0, sizeof *tr);
        uint8_t plan_node[1u << DEPTH];
        for (uint32_t p = 0; p < (1u << DEPTH); ++p) {   /* layer 0: dedup (slot, rootHold) */
            uint32_t n = 0;
            while (n < tr->count[0] && !(tr->nodes[0][n].slot == pslot[p][0] && tr->nodes[0][n].root_hold == proot[p])) ++n;
            if (n == tr->count[0]) {
                tr->nodes[0][n].slot = pslot[p][0];
                tr->nodes[0][n].root_hold = proot[p];
                tr->nodes[0][n].held_slot = pheld[p][0];
                tr->count[0]++;
            }
            plan_node[p] = (uint8_t)n;
        }
        for (uint32_t l = 1; l < DEPTH; ++l) {
            uint8_t next_node[1u << DEPTH];
            memset(next_node, 0, sizeof next_node);
            for (uint32_t par = 0; par < tr->count[l - 1]; ++par) {
                tr->nodes[l - 1][par].cbeg = tr->count[l];
                for (uint32_t p = 0; p < (1u << DEPTH); ++p) {
                    if (plan_node[p] != par) continue;
                    uint32_t n = tr->nodes[l - 1][par].cbeg;
                    while (n < tr->count[l] && tr->nodes[l][n].slot != pslot[p][l]) ++n;
                    if (n == tr->count[l]) {
                        tr->nodes[l][n].slot = pslot[p][l];
                        tr->nodes[l][n].parent = (uint8_t)par;
                        tr->nodes[l][n].held_slot = pheld[p][l];
                        tr->count[l]++;
                    }
                    next_node[p] = (uint8_t)n;
                }
                tr->nodes[l - 1][par].cend = tr->count[l];
            }
            memcpy(plan_node, next_node, sizeof plan_node);
        }
    }
}

static void ensure_ready(void) {
    if (g_ready) return;
    build_shapes();
    build_placements();
    build_trees();
    g_ready = 1;
}

/* ------------------------------------------------------ board2.hpp --- */
typedef struct { uint32_t c[W]; } board_t;

static uint32_t column_of(uint16_t cols, int col0, int x) {      /* board2.hpp:165-168 */
    uint32_t const d = (uint32_t)(x - col0);
    return d < 4 ? ((uint32_t)cols >> (4 * d)) & 0xFu : 0u;
}
static int column_top(uint32_t col) { return ctz32(col | FLOOR); }   /* board2.hpp:174 */
static int col_height(uint32_t col) { return H - column_top(col); } /* board2.hpp:127-129 */

/* board2.hpp:306-320: spawn collision and drop distance in one pass */
static int board_fit(board_t const* b, uint16_t cols, int col0, int* drop) {
    uint32_t hit = 0; int min_drop = H;
    for (int x = 0; x < W; ++x) {
        uint32_t const nib = column_of(cols, col0, x);
        hit |= b->c[x] & nib;
        int const low = bitw32(nib) - 1;
        uint32_t const mask = ~((1u << (low + 1)) - 1u);
        int const d = column_top(b->c[x] & mask) - low - 1;
        if (nib != 0 && d < min_drop) min_drop = d;
    }
    *drop = min_drop;
    return hit == 0;
}

/* board2.hpp:211-234,333-342: clear full rows, return how many */
static int board_clear(board_t* b) {
    uint32_t full = FIELD;
    for (int x = 0; x < W; ++x) full &= b->c[x];
    if (full == 0) return 0;
    for (int x = 0; x < W; ++x) {
        uint32_t col = b->c[x], fl = full;
        int const n = popc32(full);
        for (int i = 0; i < n; ++i) {
            uint32_t const row = fl & (~fl + 1u);
            uint32_t const above = col & (row - 1u);
            uint32_t const below = col & ~((row << 1) - 1u);
            col = (above << 1) | below;
            fl ^= row;
        }
        b->c[x] = col;
    }
    return popc32(full);
}

/* search.hpp:61-70 (apply): fit, place at the drop distance, clear rows */
static int apply(board_t const* b, uint16_t cols, int col0, board_t* out, int* cleared) {
    int drop;
    if (!board_fit(b, cols, col0, &drop)) return 0;
    for (int x = 0; x < W; ++x) out->c[x] = b->c[x] | (column_of(cols, col0, x) << drop);   /* board2.hpp:322-327 */
    *cleared = board_clear(out);
    return 1;
}

/* ---------------------------------------------- tetris_engine.hpp --- */
typedef struct {
    board_t board;
    uint8_t queue[QUEUE];
    uint8_t held;
    uint8_t over;
    uint8_t bag[7];
    uint32_t bag_pos;
    rng_t rng;
} engine_t;

static uint8_t draw_piece(engine_t* e) {                 /* tetris_engine.hpp:116-129 */
    if (e->bag_pos > 0) return e->bag[--e->bag_pos];
    for (int i = 0; i < 7; ++i) e->bag[i] = (uint8_t)i;
    for (uint32_t i = 6; i > 0; --i) {
        uint32_t const j = (uint32_t)(rng_next(&e->rng) % (uint64_t)(i + 1));
        uint8_t const t = e->bag[i]; e->bag[i] = e->bag[j]; e->bag[j] = t;
    }
    e->bag_pos = 6;
    return e->bag[6];
}

/* tetris_engine.hpp:159-161 with board2.hpp:241-256: can the current piece spawn TOP at (3,0)? */
static void update_game_over(engine_t* e) {
    oshape_t const s = SHAPES[e->queue[0]][0];
    int const col0 = 3 + s.left;
    uint32_t hit = 0;
    for (int x = 0; x < W; ++x) hit |= e->board.c[x] & column_of(s.cols, col0, x);
    e->over = hit != 0;
}

static void engine_reset(engine_t* e, uint64_t seed) {   /* tetris_engine.hpp:103-114 */
    memset(e, 0, sizeof *e);
    e->held = NO_PIECE;
    rng_seed(&e->rng, seed);
    for (int i = 0; i < QUEUE; ++i) e->queue[i] = draw_piece(e);
    update_game_over(e);
}

static void advance_queue(engine_t* e) {                 /* tetris_engine.hpp:131-135 */
    for (int i = 1; i < QUEUE; ++i) e->queue[i - 1] = e->queue[i];
    e->queue[QUEUE - 1] = draw_piece(e);
}

static void engine_hold(engine_t* e) {                   /* tetris_engine.hpp:148-157 */
    if (e->held == NO_PIECE) { e->held = e->queue[0]; advance_queue(e); }
    else { uint8_t const t = e->held; e->held = e->queue[0]; e->queue[0] = t; }
    update_game_over(e);
}

/* tetris_engine.hpp:137-146 (dropLocation = board2.hpp:262-279 at y=0); returns -1 for DIED */
static int engine_place(engine_t* e, int orient, int x) {
    oshape_t const s = SHAPES[e->queue[0]][orient];
    int const col0 = x + s.left;
    int min_drop = H;
    for (int c = 0; c < W; ++c) {
        uint32_t const nib = column_of(s.cols, col0, c);
        int const low = bitw32(nib) - 1;
        uint32_t const mask = ~((1u << (low + 1)) - 1u);
        int const d = column_top(e->board.c[c] & mask) - low - 1;
        if (nib != 0 && d < min_drop) min_drop = d;
    }
    for (int c = 0; c < W; ++c) e->board.c[c] |= column_of(s.cols, col0, c) << min_drop;
    int const cleared = board_clear(&e->board);
    advance_queue(e);
    update_game_over(e);
    return e->over ? -1 : cleared;
}

/* ---------------------------------------- v11 value model (FP32) --- */
/* v_board_metrics.hpp:41-56: sum of set-bit indices via 5 bit planes */
static uint32_t sum_set_bit_indices(uint32_t c) {
    /* HOLE_DEPTH_PLANES[b]: the rows y < 23 whose index has bit b set */
    static const uint32_t PLANES[5] = {0x2AAAAAu, 0x4CCCCCu, 0x70F0F0u, 0x00FF00u, 0x7F0000u};
    uint32_t s = 0;
    for (uint32_t b = 0; b < 5; ++b) s += (1u << b) * (uint32_t)popc32(c & PLANES[b]);
    return s;
}

typedef struct { uint32_t holes, hole_depths, max_height, wells; int32_t surf_sq; } board_ints_t;

/* v_board_metrics.hpp:130-225: the integer board metrics v11 reads */
static board_ints_t board_ints(board_t const* b) {
    board_ints_t r = {0, 0, 0, 0, 0};
    int h[W];
    for (int x = 0; x < W; ++x) h[x] = col_height(b->c[x]);
    for (int x = 0; x < W; ++x) {
        uint32_t const col = b->c[x];
        r.holes += (uint32_t)(h[x] - popc32(col));                        /* :130-136 */
        if ((uint32_t)h[x] > r.max_height) r.max_height = (uint32_t)h[x]; /* :146-150 */
        if (x > 0) { int const d = h[x] - h[x - 1]; r.surf_sq += d * d; } /* :152-165 */
        uint32_t const n = (uint32_t)popc32(col);                         /* :177-189 */
        uint32_t const s = sum_set_bit_indices(col);
        r.hole_depths += ((H - 1) * n + n * (n + 1) / 2) - (s + n * n);
        int well;                                                         /* :204-225 */
        if (x == 0) well = h[1] >= h[0] + 3;
        else if (x == W - 1) well = h[W - 2] >= h[W - 1] + 3;
        else well = h[x - 1] >= h[x] + 3 && h[x + 1] >= h[x] + 3;
        r.wells += (uint32_t)well;
    }
    return r;
}

static float fsqrt_ref(float x) { return x <= 0.0f ? 0.0f : sqrtf(x); }   /* v_board_metrics.hpp:23-37 */

/* model_v11.hpp:63-91: the 10 inputs */
static void extract_inputs(uint32_t clear_bits, board_t const* b, int held_is_i, float in[NIN]) {
    for (int k = 0; k < 4; ++k) in[k] = (float)((clear_bits >> (8 * k)) & 0xFFu) * 0.25f;
    board_ints_t const m = board_ints(b);
    in[4] = fsqrt_ref((float)m.surf_sq) / 100.0f;
    in[5] = (float)m.holes / 20.0f;
    in[6] = (float)m.hole_depths / 200.0f;
    in[7] = (float)m.max_height;
    in[8] = held_is_i ? 1.0f : 0.0f;
    in[9] = (float)m.wells / 5.0f;
}

/* The value network: the v11 inputs through dense layers (utility.hpp:29-46:
 * per output unit, bias first, then inputs ascending; weights [out][in] then
 * [out] biases per layer). v11 (model_v11.hpp:166-180) is h1 = 8, h2 = 0:
 * 10 -> 8 ReLU -> 1. The widened architecture is h1 = h2 = 64:
 * 10 -> 64 ReLU -> 64 ReLU -> 1. */
#define MAXH 64
typedef struct { float const* w; uint32_t h1, h2; } net_t;

static uint32_t net_params(uint32_t h1, uint32_t h2) {
    return h2 ? NIN * h1 + h1 + h1 * h2 + h2 + h2 + 1 : NIN * h1 + h1 + h1 + 1;
}

static void dense(float const* in, uint32_t n_in, float const* w, uint32_t n_out, int relu, float* out) {
    for (uint32_t o = 0; o < n_out; ++o) {
        float v = w[n_in * n_out + o];
        for (uint32_t i = 0; i < n_in; ++i) v += in[i] * w[o * n_in + i];
        out[o] = relu ? ((0.0f < v) ? v : 0.0f) : v;  /* std::max<float>(0, v) */
    }
}

static float forward(float const in[NIN], net_t const* net) {
    float h1[MAXH], h2[MAXH], out;
    dense(in, NIN, net->w, net->h1, 1, h1);
    float const* w2 = net->w + NIN * net->h1 + net->h1;
    if (!net->h2) {
        dense(h1, net->h1, w2, 1, 0, &out);
        return out;
    }
    dense(h1, net->h1, w2, net->h2, 1, h2);
    dense(h2, net->h2, w2 + net->h1 * net->h2 + net->h2, 1, 0, &out);
    return out;
}

static float evaluate(uint32_t clear_bits, board_t const* b, int held_is_i, net_t const* net) {
    float in[NIN];
    extract_inputs(clear_bits, b, held_is_i, in);
    return forward(in, net);
}

/* ------------------------------------------------- beam.hpp search --- */
static uint32_t ordered_bits(float v) {                   /* beam.hpp:204-207 */
    uint32_t u; memcpy(&u, &v, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
static float ordered_bits_inv(uint32_t s) {               /* beam.hpp:209-211 */
    uint32_t const u = (s & 0x80000000u) ? (s ^ 0x80000000u) : ~s;
    float f; memcpy(&f, &u, 4); return f;
}

/* beam.hpp:244-265: K rounds of "max non-zero score, lowest slot on ties" */
static uint32_t select_top(uint32_t* scores, uint32_t n, uint32_t k, uint32_t* out_slot, uint32_t* out_score) {
    uint32_t count = 0;
    for (; count < k; ++count) {
        uint32_t best = 0, best_slot = 0;
        for (uint32_t i = 0; i < n; ++i) if (scores[i] > best) { best = scores[i]; best_slot = i; }
        if (best == 0) break;
        out_slot[count] = best_slot; out_score[count] = best;
        scores[best_slot] = 0;
    }
    return count;
}

typedef struct {
    board_t board[32];
    uint32_t clears[32];
    uint32_t score[32];
    uint8_t node[32];
    uint8_t root_rank[32];
} frontier_t;

typedef struct { int orient, x, hold; float value; int none; } result_t;

static uint32_t clear_bump(int cleared) { return cleared == 0 ? 0u : 1u << (8 * (cleared - 1)); }  /* model_defs.hpp:37-43 */

/* beam.hpp:484-570 (search_move_beam) with the stages of beam.hpp:283-470 */
/* top2 (may be NULL) receives the best and the second-best key of the final argmax
 * (leaf keys and the dead-end fallbacks alike): diagnostics for divergence triage */
static result_t search_move_beam(engine_t const* g, net_t const* w, uint64_t* evals, uint64_t* top2) {
    result_t res = {0, 0, 0, -INFINITY, 1};
    if (g->over) return res;
    enum { ROOT_SLOTS = 2 * MP, MID_SLOTS = 32 * 2 * MP, LEAF_ORDERS = 32 * 2 * MP, SPAN = LEAF_ORDERS + 16 };

    uint8_t slot[NSLOTS];                                 /* beam.hpp:226-237 */
    slot[0] = g->held; slot[1] = g->queue[0];
    for (int i = 0; i < DEPTH; ++i) slot[2 + i] = g->queue[1 + i];
    tree_t const* tr = &TREES[g->held == NO_PIECE ? 1 : 0];
    board_t const board = g->board;

    /* stage 0: score_roots, beam.hpp:283-301 */
    uint32_t root_scores[ROOT_SLOTS];
    memset(root_scores, 0, sizeof root_scores);
    for (uint32_t gi = 0; gi < tr->count[0]; ++gi) {
        node_t const* nd = &tr->nodes[0][gi];
        uint8_t const p0 = slot[nd->slot];
        int const held_i = nd->held_slot == HELD_NONE ? 0 : slot[nd->held_slot] == 0;
        for (uint32_t i0 = 0; i0 < NPLACE[p0]; ++i0) {
            board_t nb; int cl;
            placement_t const pl = PLACEMENTS[p0][i0];
            if (apply(&board, pl.cols, pl.col0, &nb, &cl)) {
                ++*evals;
                root_scores[gi * MP + i0] = ordered_bits(evaluate(clear_bump(cl), &nb, held_i, w));
            }
        }
    }
    uint32_t top_root_slot[16], top_root_score[16];
    uint32_t const root_count = select_top(root_scores, ROOT_SLOTS, KS[0], top_root_slot, top_root_score);
    if (root_count == 0) return res;

    uint64_t best_key = 0, second_key = 0;
#define CONSIDER(sc, ord) do { uint64_t const k_ = ((uint64_t)(sc) << 32) | (uint64_t)(SPAN - (ord)); \
    if (k_ > best_key) { second_key = best_key; best_key = k_; } else if (k_ > second_key) second_key = k_; } while (0)

    frontier_t kept[2];
    uint32_t cur = 0, kept_count = root_count;
    for (uint32_t k = 0; k < root_count; ++k) {           /* seed_frontier, beam.hpp:307-329 */
        uint32_t const gi = top_root_slot[k] / MP;
        placement_t const pl = PLACEMENTS[slot[tr->nodes[0][gi].slot]][top_root_slot[k] % MP];
        int cl;
        apply(&board, pl.cols, pl.col0, &kept[0].board[k], &cl);
        kept[0].clears[k] = clear_bump(cl);
        kept[0].score[k] = top_root_score[k];
        kept[0].node[k] = (uint8_t)gi;
        kept[0].root_rank[k] = (uint8_t)k;
    }

    uint32_t mid_scores[MID_SLOTS];
    for (uint32_t level = 1; level + 1 < DEPTH; ++level) {
        frontier_t* const f = &kept[cur];
        frontier_t* const nx = &kept[cur ^ 1];
        int has_child[32];
        memset(mid_scores, 0, sizeof mid_scores);          /* score_mid_level, beam.hpp:337-372 */
        for (uint32_t k = 0; k < 32; ++k) has_child[k] = 0;
        for (uint32_t k = 0; k < kept_count; ++k) {
            node_t const* pn = &tr->nodes[level - 1][f->node[k]];
            for (uint32_t ci = pn->cbeg; ci < pn->cend; ++ci) {
                node_t const* cn = &tr->nodes[level][ci];
                uint8_t const p = slot[cn->slot];
                int const held_i = cn->held_slot == HELD_NONE ? 0 : slot[cn->held_slot] == 0;
                uint32_t const base = (k * 2 + (ci - pn->cbeg)) * MP;
                for (uint32_t i = 0; i < NPLACE[p]; ++i) {
                    board_t nb; int cl;
                    placement_t const pl = PLACEMENTS[p][i];
                    if (!apply(&f->board[k], pl.cols, pl.col0, &nb, &cl)) continue;
                    ++*evals;
                    mid_scores[base + i] = ordered_bits(evaluate(f->clears[k] + clear_bump(cl), &nb, held_i, w));
                    has_child[k] = 1;
                }
            }
        }
        uint32_t sel_slot[32], sel_score[32];
        uint32_t const next_count = select_top(mid_scores, MID_SLOTS, KS[level], sel_slot, sel_score);
        for (uint32_t k = 0; k < kept_count; ++k)          /* beam.hpp:549-551 */
            if (!has_child[k]) CONSIDER(f->score[k], LEAF_ORDERS + f->root_rank[k]);
        for (uint32_t j = 0; j < next_count; ++j) {         /* advance_frontier, beam.hpp:379-403 */
            uint32_t const k = sel_slot[j] / (2 * MP);
            node_t const* pn = &tr->nodes[level - 1][f->node[k]];
            uint32_t const ci = pn->cbeg + (sel_slot[j] / MP) % 2;
            placement_t const pl = PLACEMENTS[slot[tr->nodes[level][ci].slot]][sel_slot[j] % MP];
            int cl;
            apply(&f->board[k], pl.cols, pl.col0, &nx->board[j], &cl);
            nx->clears[j] = f->clears[k] + clear_bump(cl);
            nx->score[j] = sel_score[j];
            nx->node[j] = (uint8_t)ci;
            nx->root_rank[j] = f->root_rank[k];
        }
        cur ^= 1;
        kept_count = next_count;
    }

    frontier_t* const f = &kept[cur];                      /* expand_leaves, beam.hpp:407-443 */
    for (uint32_t j = 0; j < kept_count; ++j) {
        node_t const* ln = &tr->nodes[DEPTH - 2][f->node[j]];
        for (uint32_t ci = ln->cbeg; ci < ln->cend; ++ci) {
            node_t const* cn = &tr->nodes[DEPTH - 1][ci];
            uint8_t const p = slot[cn->slot];
            int const held_i = cn->held_slot == HELD_NONE ? 0 : slot[cn->held_slot] == 0;
            uint32_t const base = (j * 2 + (ci - ln->cbeg)) * MP;
            int expanded = 0;
            for (uint32_t i = 0; i < NPLACE[p]; ++i) {
                board_t nb; int cl;
                placement_t const pl = PLACEMENTS[p][i];
                if (!apply(&f->board[j], pl.cols, pl.col0, &nb, &cl)) continue;
                expanded = 1;
                ++*evals;
                CONSIDER(ordered_bits(evaluate(f->clears[j] + clear_bump(cl), &nb, held_i, w)), base + i);
            }
            if (!expanded) CONSIDER(f->score[j], base);
        }
    }
#undef CONSIDER

    /* decode_move, beam.hpp:450-470 */
    uint32_t const order = SPAN - (uint32_t)(best_key & 0xFFFFFFFFull);
    uint32_t const rank = order >= LEAF_ORDERS ? order - LEAF_ORDERS : f->root_rank[order / (2 * MP)];
    node_t const* rn = &tr->nodes[0][top_root_slot[rank] / MP];
    placement_t const pl0 = PLACEMENTS[slot[rn->slot]][top_root_slot[rank] % MP];
    res.orient = pl0.orient; res.x = pl0.x; res.hold = rn->root_hold;
    res.value = ordered_bits_inv((uint32_t)(best_key >> 32));
    res.none = res.value == -INFINITY;                     /* search.hpp:41 */
    if (top2) { top2[0] = best_key; top2[1] = second_key; }
    return res;
}

/* ------------------------------------------- stats_v4 + score_v1 --- */
typedef struct {
    uint32_t pieces, lines;
    uint64_t clears[5];
    uint64_t sum_max_height, sum_hole_depths;
} stats_t;

/* tetris_stats.hpp:19-23 with metrics.hpp:196-229 (the metrics score_v1 reads) */
static void stats_advance(stats_t* s, board_t const* b, uint32_t lines) {
    board_ints_t const m = board_ints(b);
    s->pieces++;
    s->lines += lines;
    s->clears[lines]++;
    s->sum_max_height += m.max_height;
    s->sum_hole_depths += m.hole_depths;
}

static double score_v1(stats_t const* s) {                /* score_v1.hpp:8-34 */
    static const double PAYOUTS[5] = {0.0, 0.2, 0.8, 2.0, 10.0};
    double clear_bonus = 0;
    for (int k = 1; k < 5; ++k) clear_bonus += PAYOUTS[k] * (double)s->clears[k];
    double const survival = 0.02 * (double)s->pieces;
    double const avg_max = (double)s->sum_max_height / (double)s->pieces;
    double const hpen = ((avg_max - 12.0) < 0.0 ? 0.0 : (avg_max - 12.0)) * 1.0;
    double const dpen = ((double)s->sum_hole_depths / (double)s->pieces) * 1.5;
    return clear_bonus + survival - hpen - dpen;
}

/* ------------------------------------------------------- C ABI ------ */
/* model_eval_host.cpp:35-51: one game, optional per-move trace (hold, orientation, x+2) */
static int play_net(net_t const* w, uint64_t seed, uint32_t max_moves, float* score, uint32_t* pieces,
                    uint32_t* lines, uint64_t* evals, uint8_t* trace, uint32_t* n_moves, uint32_t* board_out,
                    uint64_t* keys) {
    ensure_ready();
    engine_t g; engine_reset(&g, seed);
    stats_t st; memset(&st, 0, sizeof st);
    uint64_t ev = 0; uint32_t moves = 0;
    for (uint32_t i = 0; i < max_moves && !g.over; ++i) {
        result_t const r = search_move_beam(&g, w, &ev, keys ? keys + 2 * moves : NULL);
        if (r.none) break;
        if (trace) { trace[3 * moves] = (uint8_t)r.hold; trace[3 * moves + 1] = (uint8_t)r.orient; trace[3 * moves + 2] = (uint8_t)(r.x + 2); }
        ++moves;
        if (r.hold) engine_hold(&g);
        int const cl = engine_place(&g, r.orient, r.x);
        if (cl < 0) break;
        stats_advance(&st, &g.board, (uint32_t)cl);
    }
    *score = st.pieces == 0 ? -1.0e6f : (float)score_v1(&st);
    *pieces = st.pieces; *lines = st.lines;
    if (evals) *evals = ev;
    if (n_moves) *n_moves = moves;
    if (board_out) for (int x = 0; x < W; ++x) board_out[x] = g.board.c[x];
    return 0;
}

int ta3o_play(float const* w, uint64_t seed, uint32_t max_moves, float* score, uint32_t* pieces, uint32_t* lines,
              uint64_t* evals, uint8_t* trace, uint32_t* n_moves, uint32_t* board_out) {
    net_t const net = {w, NHID, 0};
    return play_net(&net, seed, max_moves, score, pieces, lines, evals, trace, n_moves, board_out, NULL);
}

/* ta3o_play plus, per searched move, the best and second-best key of the final argmax
 * (keys: 2 x max_moves; (ordered value bits << 32) | (span - order)) */
int ta3o_play_keys(float const* w, uint64_t seed, uint32_t max_moves, float* score, uint32_t* pieces,
                   uint32_t* lines, uint64_t* evals, uint8_t* trace, uint32_t* n_moves, uint64_t* keys) {
    net_t const net = {w, NHID, 0};
    return play_net(&net, seed, max_moves, score, pieces, lines, evals, trace, n_moves, NULL, keys);
}

/* one game of a dense value network with hidden widths h1, h2 (h2 = 0: one hidden layer) */
int ta3o_play_net(float const* w, uint32_t h1, uint32_t h2, uint64_t seed, uint32_t max_moves, float* score,
                  uint32_t* pieces, uint32_t* lines, uint64_t* evals, uint8_t* trace, uint32_t* n_moves,
                  uint32_t* board_out) {
    if (h1 == 0 || h1 > MAXH || h2 > MAXH) return 1;
    net_t const net = {w, h1, h2};
    return play_net(&net, seed, max_moves, score, pieces, lines, evals, trace, n_moves, board_out, NULL);
}

uint32_t ta3o_net_params(uint32_t h1, uint32_t h2) { return net_params(h1, h2); }

/* ModelEvaluator::eval_host semantics batched over models, model-major outputs */
int ta3o_eval(float const* w, uint32_t num_models, uint64_t const* seeds, uint32_t num_games, uint32_t max_moves,
              float* score_out, uint32_t* pieces_out, uint32_t* lines_out, uint64_t* evals_total) {
    uint64_t tot = 0;
    for (uint32_t m = 0; m < num_models; ++m)
        for (uint32_t gi = 0; gi < num_games; ++gi) {
            uint64_t e = 0; float s; uint32_t p, l;
            ta3o_play(w + (size_t)m * NPARAMS, seeds[gi], max_moves, &s, &p, &l, &e, 0, 0, 0);
            size_t const i = (size_t)m * num_games + gi;
            score_out[i] = s;
            if (pieces_out) pieces_out[i] = p;
            if (lines_out) lines_out[i] = l;
            tot += e;
        }
    if (evals_total) *evals_total = tot;
    return 0;
}

typedef struct {
    float const* w; uint32_t h1, h2; uint64_t const* seeds; uint32_t num_models, num_games, max_moves;
    float* score; uint32_t* pieces; uint32_t* lines;
    uint64_t next, evals; pthread_mutex_t mu;
} mt_job_t;

static void* mt_worker(void* arg) {
    mt_job_t* j = (mt_job_t*)arg;
    uint64_t const total = (uint64_t)j->num_models * j->num_games;
    uint64_t local = 0;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        uint64_t const i = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (i >= total) break;
        uint64_t e = 0; float s; uint32_t p, l;
        net_t const net = {j->w + (i / j->num_games) * net_params(j->h1, j->h2), j->h1, j->h2};
        play_net(&net, j->seeds[i % j->num_games], j->max_moves, &s, &p, &l, &e, 0, 0, 0, 0);
        j->score[i] = s;
        if (j->pieces) j->pieces[i] = p;
        if (j->lines) j->lines[i] = l;
        local += e;
    }
    pthread_mutex_lock(&j->mu);
    j->evals += local;
    pthread_mutex_unlock(&j->mu);
    return 0;
}

/* the same batch spread over `threads` host threads, (model, game) pairs pulled from a shared ticket */
static int eval_net_mt(float const* w, uint32_t h1, uint32_t h2, uint32_t num_models, uint64_t const* seeds,
                       uint32_t num_games, uint32_t max_moves, uint32_t threads, float* score_out,
                       uint32_t* pieces_out, uint32_t* lines_out, uint64_t* evals_total) {
    ensure_ready();
    mt_job_t j = {w, h1, h2, seeds, num_models, num_games, max_moves, score_out, pieces_out, lines_out, 0, 0,
                  PTHREAD_MUTEX_INITIALIZER};
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], 0, mt_worker, &j);
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], 0);
    if (evals_total) *evals_total = j.evals;
    return 0;
}

int ta3o_eval_mt(float const* w, uint32_t num_models, uint64_t const* seeds, uint32_t num_games, uint32_t max_moves,
                 uint32_t threads, float* score_out, uint32_t* pieces_out, uint32_t* lines_out, uint64_t* evals_total) {
    return eval_net_mt(w, NHID, 0, num_models, seeds, num_games, max_moves, threads, score_out, pieces_out, lines_out,
                       evals_total);
}

/* the batch for a dense network with hidden widths h1, h2 */
int ta3o_eval_net_mt(float const* w, uint32_t h1, uint32_t h2, uint32_t num_models, uint64_t const* seeds,
                     uint32_t num_games, uint32_t max_moves, uint32_t threads, float* score_out, uint32_t* pieces_out,
                     uint32_t* lines_out, uint64_t* evals_total) {
    if (h1 == 0 || h1 > MAXH || h2 > MAXH) return 1;
    return eval_net_mt(w, h1, h2, num_models, seeds, num_games, max_moves, threads, score_out, pieces_out, lines_out,
                       evals_total);
}

uint32_t ta3o_placements(uint32_t piece, uint8_t* orient, int8_t* x, uint16_t* cols, int8_t* col0) {
    ensure_ready();
    for (uint32_t i = 0; i < NPLACE[piece]; ++i) {
        orient[i] = PLACEMENTS[piece][i].orient; x[i] = PLACEMENTS[piece][i].x;
        cols[i] = PLACEMENTS[piece][i].cols; col0[i] = PLACEMENTS[piece][i].col0;
    }
    return NPLACE[piece];
}

void ta3o_plan_tree(uint32_t held_empty, uint32_t* counts, uint8_t* nodes6) {
    ensure_ready();
    tree_t const* tr = &TREES[held_empty ? 1 : 0];
    for (uint32_t l = 0; l < DEPTH; ++l) {
        counts[l] = tr->count[l];
        for (uint32_t n = 0; n < (1u << DEPTH); ++n) {
            node_t const* nd = &tr->nodes[l][n];
            uint8_t* o = nodes6 + (l * (1u << DEPTH) + n) * 6;
            o[0] = nd->slot; o[1] = nd->parent; o[2] = nd->cbeg; o[3] = nd->cend; o[4] = nd->root_hold; o[5] = nd->held_slot;
        }
    }
}

void ta3o_piece_queue(uint64_t seed, uint32_t* queue6) {
    ensure_ready();
    engine_t g; engine_reset(&g, seed);
    for (int i = 0; i < QUEUE; ++i) queue6[i] = g.queue[i];
}

/* the first n pieces the engine deals for a seed (queue then bag), ta3_sim piece supply */
void ta3o_piece_sequence(uint64_t seed, uint32_t n, uint8_t* out) {
    ensure_ready();
    engine_t g; engine_reset(&g, seed);
    for (uint32_t i = 0; i < n; ++i) { out[i] = g.queue[0]; advance_queue(&g); }
}

void ta3o_simulate_seeds(uint64_t seed, uint32_t games, uint64_t* out) {   /* model_eval.hpp:84-103 */
    rng_t r; rng_seed(&r, seed);
    for (uint32_t i = 0; i < games; ++i) out[i] = rng_next(&r);
}

float ta3o_evaluate(float const* w, uint32_t const* cols10, uint32_t clear_bits, int held_is_i, float* features10) {
    ensure_ready();
    board_t b; memcpy(b.c, cols10, sizeof b.c);
    extract_inputs(clear_bits, &b, held_is_i, features10);
    net_t const net = {w, NHID, 0};
    return forward(features10, &net);
}

int ta3o_apply(uint32_t const* cols10, uint32_t piece, uint32_t index, uint32_t* out10, uint32_t* cleared) {
    ensure_ready();
    board_t b, nb; int cl = 0;
    memcpy(b.c, cols10, sizeof b.c);
    placement_t const pl = PLACEMENTS[piece][index];
    int const ok = apply(&b, pl.cols, pl.col0, &nb, &cl);
    memcpy(out10, ok ? nb.c : b.c, sizeof nb.c);
    *cleared = ok ? (uint32_t)cl : 0u;
    return ok;
}

/* integer board metrics, for known-answer tests (holes, hole depths, max height, wells, surface sum) */
void ta3o_board_ints(uint32_t const* cols10, uint32_t* out5) {
    board_t b; memcpy(b.c, cols10, sizeof b.c);
    board_ints_t const m = board_ints(&b);
    out5[0] = m.holes; out5[1] = m.hole_depths; out5[2] = m.max_height; out5[3] = m.wells; out5[4] = (uint32_t)m.surf_sq;
}

uint32_t ta3o_num_params(void) { return NPARAMS; }
