// Host build of eval_core.h for the CPU tests only (tests/test_core_host.py):
// it lets the incremental candidate path be checked against the oracle on
// many boards without a GPU. The product library never contains this file.
#include "eval_core.h"

#include <algorithm>
#include <utility>

namespace {
struct HostW {
    float const* p;
    float operator()(int i) const { return p[i]; }
};
} // namespace

extern "C" {

uint32_t ta3bt_rec_words() { return uint32_t(ta3b::REC_WORDS); }

void ta3bt_build_record(uint32_t const* b10, uint32_t clears, float const* w97, uint32_t* rec) {
    uint32_t b[ta3b::W];
    for (int x = 0; x < ta3b::W; ++x) b[x] = b10[x];
    ta3b::build_record(b, clears, HostW{w97}, rec);
}

// 0 = fast path evaluated, 1 = deferred to the full path
int ta3bt_fast(uint32_t const* rec, uint32_t piece, uint32_t idx, int held, float const* w97, float* value,
               float* dbg) {
    ta3b::FastW fw;
    ta3b::load_fast_weights(HostW{w97}, fw);
    ta3b::RecView r;
    for (int o = 0; o < ta3b::NHID; ++o) __builtin_memcpy(&r.P[o], &rec[ta3b::R_P + o], 4);
    r.tot = rec[ta3b::R_TOT];
    r.hd = rec[ta3b::R_HD];
    r.rc0 = rec[ta3b::R_RC];
    r.rc1 = rec[ta3b::R_RC + 1];
    r.rc2 = rec[ta3b::R_RC + 2];
    ta3b::PlaceFast const pf = ta3b::FAST.place[piece][idx];
    ta3b::span_of(rec, int((pf.m >> 27) & 0xFu), r.h4, r.hm4);
    r.combo = rec[ta3b::R_COMBO + ((pf.m >> 16) & 63u)];
    return ta3b::fast_eval<ta3b::MLP_SCALAR>(r, pf, held != 0, fw, *value, dbg);
}

// legality; value / cleared / resulting board of the full path
int ta3bt_full(uint32_t const* b10, uint32_t clears, uint32_t piece, uint32_t idx, int held, float const* w97,
               float* value, uint32_t* cleared, uint32_t* out10) {
    uint32_t b[ta3b::W], nb[ta3b::W];
    for (int x = 0; x < ta3b::W; ++x) b[x] = b10[x];
    ta3b::Place const pl = ta3b::TABLES.place[piece][idx];
    int cl = 0;
    if (!ta3b::apply_full(b, pl.cols, pl.col0, nb, cl)) return 0;
    ta3b::BoardInts const bi = ta3b::board_ints(nb);
    *value = ta3b::value_full(clears + ta3b::clear_bump(cl), bi, held != 0, HostW{w97});
    *cleared = uint32_t(cl);
    for (int x = 0; x < ta3b::W; ++x) out10[x] = nb[x];
    return 1;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Host emulation of the kernel's search over the same core: records per kept
// node, fast path with full-path fallback, the root record built the way the
// warp builds it (one piece per "lane"). Plays whole games so the CPU tests can
// compare move traces with the oracle.
#include <cstring>
#include <vector>

namespace {

using namespace ta3b;

struct Eng {
    uint32_t b[W];
    uint64_t s[4];
    uint32_t q[QUEUE], bag[7], bag_pos, held;
    bool over;
};

uint64_t nxt(uint64_t (&s)[4]) {
    uint64_t const r = ((s[1] * 5) << 7 | (s[1] * 5) >> 57) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return r;
}
uint32_t draw(Eng& e) {
    if (e.bag_pos > 0) return e.bag[--e.bag_pos];
    for (int i = 0; i < 7; ++i) e.bag[i] = uint32_t(i);
    for (uint32_t i = 6; i > 0; --i) {
        uint32_t const j = uint32_t(nxt(e.s) % (i + 1));
        std::swap(e.bag[i], e.bag[j]);
    }
    e.bag_pos = 6;
    return e.bag[6];
}
void gameover(Eng& e) {
    uint32_t const p = e.q[0], cols = TABLES.spawn_cols[p];
    int const c0 = TABLES.spawn_col0[p];
    uint32_t hit = 0;
    for (int i = 0; i < 4; ++i)
        if (c0 + i < W) hit |= e.b[c0 + i] & ((cols >> (4 * i)) & 0xFu);
    e.over = hit != 0;
}
void reset(Eng& e, uint64_t seed) {
    std::memset(&e, 0, sizeof e);
    for (int i = 0; i < 4; ++i) {
        seed += 0x9e3779b97f4a7c15ULL;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        e.s[i] = z ^ (z >> 31);
    }
    e.held = NO_PIECE;
    for (int i = 0; i < QUEUE; ++i) e.q[i] = draw(e);
    gameover(e);
}
void advq(Eng& e) {
    for (int i = 1; i < QUEUE; ++i) e.q[i - 1] = e.q[i];
    e.q[QUEUE - 1] = draw(e);
}

struct Node {
    uint32_t rec[REC_WORDS];
    uint32_t score, node, rank;
};

struct Cand {
    uint64_t key;
    bool legal;
};

unsigned long long g_fast_count = 0, g_defer_count = 0;

// one candidate through the kernel's paths
Cand candidate(uint32_t const* rec, int piece, int i, bool held, bool leaf, uint32_t k, uint32_t child,
               FastW const& fw, HostW const& w) {
    PlaceFast const pf = FAST.place[piece][i];
    RecView r;
    for (int o = 0; o < NHID; ++o) __builtin_memcpy(&r.P[o], &rec[R_P + o], 4);
    r.tot = rec[R_TOT]; r.hd = rec[R_HD]; r.rc0 = rec[R_RC]; r.rc1 = rec[R_RC + 1]; r.rc2 = rec[R_RC + 2];
    span_of(rec, int((pf.m >> 27) & 0xFu), r.h4, r.hm4);
    r.combo = rec[R_COMBO + ((pf.m >> 16) & 63u)];
    float v;
    bool const fast = fast_eval<MLP_SCALAR>(r, pf, held, fw, v) == FAST_OK;
    ++(fast ? g_fast_count : g_defer_count);
    if (!fast) {
        uint32_t b[W], nb[W];
        for (int x = 0; x < W; ++x) b[x] = rec[R_BOARD + x];
        Place const pl = TABLES.place[piece][i];
        int cl = 0;
        if (!apply_full(b, pl.cols, pl.col0, nb, cl)) return {0, false};
        v = value_full(rec[R_CLEARS] + clear_bump(cl), board_ints(nb), held, w);
    }
    uint32_t const pos = (k * 2u + child) * MP + uint32_t(i);
    uint32_t const low = leaf ? uint32_t(ORDER_SPAN) - pos : 0xFFFFFFFFu - pos;
    return {(uint64_t(ordered_bits(v)) << 32) | low, true};
}

void child_record(uint32_t const* prec, int piece, int i, HostW const& w, uint32_t* out) {
    uint32_t b[W], nb[W];
    for (int x = 0; x < W; ++x) b[x] = prec[R_BOARD + x];
    Place const pl = TABLES.place[piece][i];
    int cl = 0;
    apply_full(b, pl.cols, pl.col0, nb, cl);
    build_record(nb, prec[R_CLEARS] + clear_bump(cl), w, out);
}

unsigned long long g_insertions = 0, g_rounds = 0, g_levels = 0, g_cands = 0;

// insertions the warp's top-k fold performs when the keys arrive 32 per round in
// flattened order (a key is inserted when it beats the current k-th best)
void count_insertions(std::vector<uint64_t> const& keys, size_t k) {
    std::vector<uint64_t> list;
    ++g_levels;
    for (size_t r = 0; r < keys.size(); r += 32) {
        ++g_rounds;
        for (size_t l = r; l < keys.size() && l < r + 32; ++l) {
            uint64_t const thr = list.size() < k ? 0 : list[k - 1];
            if (keys[l] > thr) {
                ++g_insertions;
                list.insert(std::upper_bound(list.begin(), list.end(), keys[l], [](uint64_t a, uint64_t b) { return a > b; }), keys[l]);
                if (list.size() > k) list.pop_back();
            }
        }
    }
    g_cands += keys.size();
}

// top-k of (key) with keys unique; returns sorted descending
std::vector<uint64_t> topk(std::vector<uint64_t> keys, size_t k) {
    count_insertions(keys, k);
    std::sort(keys.begin(), keys.end(), [](uint64_t a, uint64_t b) { return a > b; });
    while (!keys.empty() && keys.back() == 0) keys.pop_back();
    if (keys.size() > k) keys.resize(k);
    return keys;
}

} // namespace

extern "C" {

void ta3bt_path_counts(unsigned long long* fast, unsigned long long* deferred) {
    *fast = g_fast_count;
    *deferred = g_defer_count;
}

void ta3bt_topk_counts(unsigned long long* ins, unsigned long long* rounds, unsigned long long* levels,
                       unsigned long long* cands) {
    *ins = g_insertions;
    *rounds = g_rounds;
    *levels = g_levels;
    *cands = g_cands;
}

// root record the way the warp builds it (each "lane" writes its own words)
void ta3bt_root_record(uint32_t const* b10, float const* w97, uint32_t* rec) {
    uint32_t b[W];
    for (int x = 0; x < W; ++x) b[x] = b10[x];
    HostW const w{w97};
    for (int lane = 0; lane < 32; ++lane) {
        ColumnData c;
        column_data(b, c);
        if (lane < W) rec[R_BOARD + lane] = b[lane];
        if (lane == 22) {
            uint32_t hb[4], hmb[4];
            span_bytes(c, hb, hmb);
            for (int q = 0; q < 4; ++q) {
                rec[R_HB + q] = hb[q];
                rec[R_HMB + q] = hmb[q];
            }
        }
        for (int id = lane; id < NCOMBO; id += 32) {
            int c0, wd;
            combo_of(id, c0, wd);
            rec[R_COMBO + id] = combo_word(c, c0, wd);
        }
        if (lane < NHID) rec[R_P + lane] = partial_word(0u, lane, w);
        if (lane >= 16 && lane < 19) rec[R_RC + lane - 16] = row_counts(b, lane - 16);
        if (lane == 20) rec[R_HD] = hole_depths_total(b);
        if (lane == 21) {
            rec[R_CLEARS] = 0;
            rec[R_TOT] = c.holes | (c.maxh << 8) | (uint32_t(c.pw[W]) << 13) | (uint32_t(c.pp[W]) << 17);
        }
    }
}

// a whole game through the kernel's algorithm; trace = 3 bytes per move
int ta3bt_play(float const* w97, uint64_t seed, uint32_t max_moves, uint8_t* trace, uint32_t* n_moves,
               uint32_t* pieces) {
    HostW const w{w97};
    FastW fw;
    load_fast_weights(w, fw);
    Eng e;
    reset(e, seed);
    uint32_t moves = 0, placed = 0;
    for (uint32_t mvi = 0; mvi < max_moves && !e.over; ++mvi) {
        uint32_t slot[NSLOTS] = {e.held, e.q[0], e.q[1], e.q[2], e.q[3], e.q[4]};
        int const tree = e.held == NO_PIECE ? 1 : 0;
        uint32_t root[REC_WORDS];
        ta3bt_root_record(e.b, w97, root);
        TreeNode const* L0 = TABLES.tree[tree][0];
        std::vector<uint64_t> keys;
        for (uint32_t g = 0; g < 2; ++g) {
            int const p = int(slot[L0[g].slot]);
            bool const hi = L0[g].held != HELD_NONE && slot[L0[g].held] == 0;
            for (int i = 0; i < TABLES.nplace[p]; ++i) keys.push_back(candidate(root, p, i, hi, false, 0, g, fw, w).key);
        }
        auto const roots = topk(keys, K0);
        if (roots.empty()) break;
        std::vector<Node> fr(roots.size());
        std::vector<uint32_t> root_slot(roots.size());
        for (size_t k = 0; k < roots.size(); ++k) {
            uint32_t const rs = 0xFFFFFFFFu - uint32_t(roots[k]);
            root_slot[k] = rs;
            uint32_t const g = rs / MP;
            child_record(root, int(slot[L0[g].slot]), int(rs % MP), w, fr[k].rec);
            fr[k].score = uint32_t(roots[k] >> 32);
            fr[k].node = g;
            fr[k].rank = uint32_t(k);
        }
        uint64_t best = 0;
        for (int level = 1; level < DEPTH; ++level) {
            bool const leaf = level == DEPTH - 1;
            std::vector<uint64_t> lk;
            std::vector<bool> has(fr.size(), false);
            for (size_t k = 0; k < fr.size(); ++k)
                for (uint32_t ch = 0; ch < 2; ++ch) {
                    TreeNode const& cn = TABLES.tree[tree][level][2 * fr[k].node + ch];
                    int const p = int(slot[cn.slot]);
                    bool const hi = cn.held != HELD_NONE && slot[cn.held] == 0;
                    bool any = false;
                    for (int i = 0; i < TABLES.nplace[p]; ++i) {
                        Cand const c = candidate(fr[k].rec, p, i, hi, leaf, uint32_t(k), ch, fw, w);
                        if (!c.legal) continue;
                        any = true;
                        if (leaf) best = c.key > best ? c.key : best;
                        else lk.push_back(c.key);
                    }
                    has[k] = has[k] || any;
                    if (leaf && !any) {
                        uint64_t const key = (uint64_t(fr[k].score) << 32) | uint64_t(ORDER_SPAN - (k * 2 + ch) * MP);
                        best = key > best ? key : best;
                    }
                }
            if (leaf) break;
            for (size_t k = 0; k < fr.size(); ++k)
                if (!has[k]) {
                    uint64_t const key = (uint64_t(fr[k].score) << 32) | uint64_t(ORDER_SPAN - (LEAF_ORDERS + fr[k].rank));
                    best = key > best ? key : best;
                }
            auto const sel = topk(lk, 32);
            std::vector<Node> nx(sel.size());
            for (size_t j = 0; j < sel.size(); ++j) {
                uint32_t const ss = 0xFFFFFFFFu - uint32_t(sel[j]);
                uint32_t const k = ss / (2 * MP), ch = (ss / MP) & 1u;
                uint32_t const cnode = 2 * fr[k].node + ch;
                int const p = int(slot[TABLES.tree[tree][level][cnode].slot]);
                child_record(fr[k].rec, p, int(ss % MP), w, nx[j].rec);
                nx[j].score = uint32_t(sel[j] >> 32);
                nx[j].node = cnode;
                nx[j].rank = fr[k].rank;
            }
            fr.swap(nx);
        }
        uint32_t const order = ORDER_SPAN - uint32_t(best);
        uint32_t const rank = order >= uint32_t(LEAF_ORDERS) ? order - LEAF_ORDERS : fr[order / (2 * MP)].rank;
        uint32_t const rs = root_slot[rank];
        uint32_t const g = rs / MP;
        Place const pl = TABLES.place[slot[L0[g].slot]][rs % MP];
        trace[3 * moves] = L0[g].root_hold;
        trace[3 * moves + 1] = pl.orient;
        trace[3 * moves + 2] = uint8_t(pl.x + 2);
        ++moves;
        if (L0[g].root_hold) {
            if (e.held == NO_PIECE) { e.held = e.q[0]; advq(e); }
            else std::swap(e.held, e.q[0]);
            gameover(e);
        }
        uint32_t const p = e.q[0];
        int cl = 0;
        uint32_t nb[W];
        apply_full(e.b, TABLES.shape_cols[p][pl.orient], pl.x + TABLES.shape_left[p][pl.orient], nb, cl);
        for (int x = 0; x < W; ++x) e.b[x] = nb[x];
        advq(e);
        gameover(e);
        if (e.over) break;
        ++placed;
    }
    *n_moves = moves;
    *pieces = placed;
    return 0;
}

} // extern "C"
