// Game geometry and search-shape tables, derived at compile time (host and
// device) from the tetromino block coordinates.
//
// These tables must equal the reference's, entry for entry, because the
// search's tie-breaks are defined over their index order:
//   * block coordinates          ta3_sim/incl/ta3/sim/pieces/piece_offsets.hpp:19-85
//   * trimmed nibble shapes      ta3_sim/incl/ta3/sim/pieces/piece_offsets.hpp:112-201
//   * deduped placement order    ta3_ai/incl/ta3/ai/search/placements.hpp:70-205
//   * hold-plan prefix trees     ta3_ai/incl/ta3/ai/search/variation_sequences.hpp:216-259,
//                                ta3_ai/incl/ta3/ai/search/beam.hpp:69-128
// The derivation below is written independently; tests/golden/tables.json
// (produced by the reference) pins its output.
#pragma once
#include <cstdint>

namespace ta3b {

constexpr int W = 10;                       // board columns
constexpr int H = 23;                       // board rows (3 hidden spawn rows), bit 0 = top
constexpr uint32_t FIELD = (1u << H) - 1u;
constexpr uint32_t FLOOR = 1u << H;         // sentinel: empty column has its top at H
constexpr int NPIECE = 7;                   // I O T S Z J L
constexpr int NO_PIECE = 7;
constexpr int QUEUE = 6;                    // current + 5 preview
constexpr int DEPTH = 4;                    // beam widths {16, 32, 32} -> 4 placed pieces
constexpr int K0 = 16, K1 = 32, K2 = 32;    // beam widths per kept level
constexpr int MP = 34;                      // max placements of one piece
constexpr int NSLOTS = DEPTH + 2;           // window slots: 0 held, 1 current, 2.. preview
constexpr int HELD_NONE = 7;
constexpr int ROOT_SLOTS = 2 * MP;          // 2 root groups x 34
constexpr int LEAF_ORDERS = K2 * 2 * MP;    // 2176
constexpr int ORDER_SPAN = LEAF_ORDERS + K0;// 2192
constexpr int NPARAMS = 97;                 // v11: 10 -> 8 (ReLU) -> 1
constexpr int NIN = 10, NHID = 8;

// Block coordinates, [piece][orientation TOP,RIGHT,BOTTOM,LEFT][block][x,y].
constexpr int8_t BLOCKS[NPIECE][4][4][2] = {
    /* I */ {{{0,1},{1,1},{2,1},{3,1}}, {{2,0},{2,1},{2,2},{2,3}}, {{0,2},{1,2},{2,2},{3,2}}, {{1,0},{1,1},{1,2},{1,3}}},
    /* O */ {{{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{2,1}}},
    /* T */ {{{1,0},{0,1},{1,1},{2,1}}, {{1,0},{1,1},{2,1},{1,2}}, {{0,1},{1,1},{2,1},{1,2}}, {{1,0},{0,1},{1,1},{1,2}}},
    /* S */ {{{1,0},{2,0},{0,1},{1,1}}, {{0,0},{0,1},{1,1},{1,2}}, {{1,1},{2,1},{1,2},{0,2}}, {{1,0},{1,1},{2,1},{2,2}}},
    /* Z */ {{{0,0},{1,0},{1,1},{2,1}}, {{2,0},{1,1},{2,1},{1,2}}, {{1,1},{0,1},{1,2},{2,2}}, {{1,0},{0,1},{1,1},{0,2}}},
    /* J */ {{{0,0},{0,1},{1,1},{2,1}}, {{1,0},{2,0},{1,1},{1,2}}, {{0,1},{1,1},{2,1},{2,2}}, {{1,0},{1,1},{0,2},{1,2}}},
    /* L */ {{{2,0},{0,1},{1,1},{2,1}}, {{1,0},{1,1},{1,2},{2,2}}, {{0,1},{1,1},{2,1},{0,2}}, {{0,0},{1,0},{1,1},{1,2}}},
};

// One placement: nibble-packed occupied columns (nibble i = board column col0+i,
// bit y = local row y), the first occupied board column, and the move it
// stands for (orientation, window x-origin).
struct Place {
    uint16_t cols;
    int8_t col0;
    uint8_t orient;
    int8_t x;
};

// Hold-plan prefix tree node: the window slot placed at this level, the slot
// sitting in hold after this level's decision, and (layer 0) the root hold flag.
struct TreeNode {
    uint8_t slot, held, root_hold, parent, cbeg, cend;
};

struct Tables {
    Place place[NPIECE][MP];
    uint8_t nplace[NPIECE];
    uint16_t spawn_cols[NPIECE];            // TOP shape, for the spawn / game-over check
    int8_t spawn_col0[NPIECE];
    uint16_t shape_cols[NPIECE][4];         // every orientation, for committing a move
    int8_t shape_left[NPIECE][4];
    TreeNode tree[2][DEPTH][16];            // [held_empty][layer][node]
    uint8_t tree_count[2][DEPTH];
};

constexpr Tables make_tables() {
    Tables t{};
    for (int p = 0; p < NPIECE; ++p) {
        uint16_t cols[4]{};
        int8_t left[4]{};
        uint8_t ncols[4]{};
        for (int o = 0; o < 4; ++o) {
            uint32_t box[4]{};
            for (int b = 0; b < 4; ++b) box[BLOCKS[p][o][b][0]] |= 1u << BLOCKS[p][o][b][1];
            int l = 0;
            while (l < 4 && box[l] == 0) ++l;
            int r = 4;
            while (r > l && box[r - 1] == 0) --r;
            uint32_t c = 0;
            for (int i = 0; i < r - l; ++i) c |= box[l + i] << (4 * i);
            cols[o] = static_cast<uint16_t>(c);
            left[o] = static_cast<int8_t>(l);
            ncols[o] = static_cast<uint8_t>(r - l);
            t.shape_cols[p][o] = cols[o];
            t.shape_left[p][o] = left[o];
        }
        t.spawn_cols[p] = cols[0];
        t.spawn_col0[p] = static_cast<int8_t>(3 + left[0]);
        // dedupe orientations by their vertically normalised column signature,
        // keeping the lowest orientation index; then every legal x-origin
        uint32_t sig[4]{};
        int nsig = 0, w = 0;
        for (int o = 0; o < 4; ++o) {
            uint32_t minbit = 32;
            for (int i = 0; i < ncols[o]; ++i) {
                uint32_t v = (cols[o] >> (4 * i)) & 0xFu;
                uint32_t b = 0;
                while (v && !((v >> b) & 1u)) ++b;
                if (v && b < minbit) minbit = b;
            }
            if (minbit == 32) minbit = 0;
            uint32_t s = ncols[o];
            for (int i = 0; i < ncols[o]; ++i) s |= (((cols[o] >> (4 * i)) & 0xFu) >> minbit) << (4 + 4 * i);
            bool dup = false;
            for (int j = 0; j < nsig; ++j) dup = dup || sig[j] == s;
            if (dup) continue;
            sig[nsig++] = s;
            for (int x = -left[o]; x <= W - left[o] - ncols[o]; ++x)
                t.place[p][w++] = Place{cols[o], static_cast<int8_t>(x + left[o]), static_cast<uint8_t>(o),
                                        static_cast<int8_t>(x)};
        }
        t.nplace[p] = static_cast<uint8_t>(w);
    }
    // hold plans: every 2^DEPTH hold/no-hold decision vector over window slots,
    // regrouped into a prefix tree (layer 0 keyed on (slot, root hold))
    for (int he = 0; he < 2; ++he) {
        uint8_t ps[16][DEPTH]{}, ph[16][DEPTH]{}, pr[16]{};
        for (int d = 0; d < 16; ++d) {
            uint8_t cur = 1, hld = 0;
            bool empty = he == 1;
            int k = 1;
            for (int i = 0; i < DEPTH; ++i) {
                bool did = false;
                if (d & (1 << i)) {
                    if (empty) { hld = cur; cur = static_cast<uint8_t>(1 + k++); empty = false; }
                    else { uint8_t tmp = cur; cur = hld; hld = tmp; }
                    did = true;
                }
                ps[d][i] = cur;
                if (i == 0) pr[d] = did;
                ph[d][i] = empty ? HELD_NONE : hld;
                if (i + 1 < DEPTH) cur = static_cast<uint8_t>(1 + k++);
            }
        }
        uint8_t pn[16]{};
        for (int d = 0; d < 16; ++d) {
            int n = 0;
            while (n < t.tree_count[he][0] && !(t.tree[he][0][n].slot == ps[d][0] && t.tree[he][0][n].root_hold == pr[d])) ++n;
            if (n == t.tree_count[he][0]) {
                t.tree[he][0][n] = TreeNode{ps[d][0], ph[d][0], pr[d], 0, 0, 0};
                ++t.tree_count[he][0];
            }
            pn[d] = static_cast<uint8_t>(n);
        }
        for (int l = 1; l < DEPTH; ++l) {
            uint8_t nn[16]{};
            for (int par = 0; par < t.tree_count[he][l - 1]; ++par) {
                t.tree[he][l - 1][par].cbeg = t.tree_count[he][l];
                for (int d = 0; d < 16; ++d) {
                    if (pn[d] != par) continue;
                    int n = t.tree[he][l - 1][par].cbeg;
                    while (n < t.tree_count[he][l] && t.tree[he][l][n].slot != ps[d][l]) ++n;
                    if (n == t.tree_count[he][l]) {
                        t.tree[he][l][n] = TreeNode{ps[d][l], ph[d][l], 0, static_cast<uint8_t>(par), 0, 0};
                        ++t.tree_count[he][l];
                    }
                    nn[d] = static_cast<uint8_t>(n);
                }
                t.tree[he][l - 1][par].cend = t.tree_count[he][l];
            }
            for (int d = 0; d < 16; ++d) pn[d] = nn[d];
        }
    }
    return t;
}

constexpr Tables TABLES = make_tables();

// Per-placement data for the incremental candidate path (16 bytes):
//   d4  byte i = 22 - lowest cell row of piece column i (i < width), 127 beyond
//   c4  byte i = cells in piece column i (i < width), 0 beyond
//   m   cells per local row r (nibble r, 16 bits) | combo id (6) << 16 | width==1 << 22
//       | has left neighbour column << 23 | has right neighbour column << 24
//       | min over columns of the highest cell row (2) << 25 | window origin c0 (4) << 27
//   s   sum_{i<w} (22 - low_i) (7) | sum_i cells_i * (22 - low_i) (7) << 7
//       | sum of squared top-row steps inside the piece (4) << 14 | top row of column 0 (2) << 18
//       | top row of the last column (2) << 20 | width (3) << 22
// A combo is one (window origin c0, width w) pair; the 34 combos index the
// per-parent table of old surface / well terms.
struct PlaceFast {
    uint32_t d4, c4, m, s;
};

constexpr int combo_id(int c0, int w) {
    return (w == 1 ? 0 : w == 2 ? 10 : w == 3 ? 19 : 27) + c0;
}
constexpr int NCOMBO = 34;

constexpr PlaceFast make_place_fast(Place p) {
    uint32_t width = 0, pr = 0;
    uint32_t low[4]{}, first[4]{}, cnt[4]{};
    for (int i = 0; i < 4; ++i) {
        uint32_t const nib = (uint32_t(p.cols) >> (4 * i)) & 0xFu;
        if (!nib) continue;
        width = uint32_t(i + 1);
        uint32_t lo = 0, fi = 3, n = 0;
        for (uint32_t r = 0; r < 4; ++r)
            if ((nib >> r) & 1u) {
                lo = r;
                if (r < fi) fi = r;
                ++n;
                pr += 1u << (4 * r);
            }
        low[i] = lo;
        first[i] = fi;
        cnt[i] = n;
    }
    uint32_t d4 = 0, c4 = 0, a1 = 0, a2 = 0, sint = 0, minfirst = 3;
    for (uint32_t i = 0; i < 4; ++i) {
        uint32_t const d = i < width ? 22u - low[i] : 127u;
        d4 |= d << (8 * i);
        c4 |= (i < width ? cnt[i] : 0u) << (8 * i);
        if (i < width) {
            a1 += 22u - low[i];
            a2 += cnt[i] * (22u - low[i]);
            if (first[i] < minfirst) minfirst = first[i];
            if (i + 1 < width) {
                int const step = int(first[i]) - int(first[i + 1]);
                sint += uint32_t(step * step);
            }
        }
    }
    int const c0 = p.col0;
    uint32_t const m = pr | (uint32_t(combo_id(c0, int(width))) << 16) | (uint32_t(width == 1) << 22) |
                       (uint32_t(c0 > 0) << 23) | (uint32_t(c0 + int(width) < W) << 24) | (minfirst << 25) |
                       (uint32_t(c0) << 27);
    uint32_t const s = a1 | (a2 << 7) | (sint << 14) | (first[0] << 18) | (first[width - 1] << 20) | (width << 22);
    return PlaceFast{d4, c4, m, s};
}

struct FastTables {
    PlaceFast place[NPIECE][MP];
};

constexpr FastTables make_fast_tables() {
    FastTables f{};
    for (int p = 0; p < NPIECE; ++p)
        for (int i = 0; i < TABLES.nplace[p]; ++i) f.place[p][i] = make_place_fast(TABLES.place[p][i]);
    return f;
}

constexpr FastTables FAST = make_fast_tables();

// adjacent piece columns' top rows differ by at most 2, so no column inside a
// piece's span can be a well (depth >= 3) right after the drop
constexpr bool span_has_no_wells() {
    for (int p = 0; p < NPIECE; ++p)
        for (int i = 0; i < TABLES.nplace[p]; ++i) {
            PlaceFast const f = FAST.place[p][i];
            uint32_t const w = (f.s >> 22) & 7u;
            for (uint32_t c = 0; c + 1 < w; ++c) {
                uint32_t const nib0 = (uint32_t(TABLES.place[p][i].cols) >> (4 * c)) & 0xFu;
                uint32_t const nib1 = (uint32_t(TABLES.place[p][i].cols) >> (4 * (c + 1))) & 0xFu;
                int f0 = 0, f1 = 0;
                while (!((nib0 >> f0) & 1u)) ++f0;
                while (!((nib1 >> f1) & 1u)) ++f1;
                if (f0 - f1 > 2 || f1 - f0 > 2) return false;
            }
        }
    return true;
}
static_assert(span_has_no_wells(), "piece columns' top rows must differ by <= 2");

// every tetromino column is one contiguous run of cells (the incremental path relies on it)
constexpr bool columns_contiguous() {
    for (int p = 0; p < NPIECE; ++p)
        for (int o = 0; o < 4; ++o)
            for (int i = 0; i < 4; ++i) {
                uint32_t const nib = (uint32_t(TABLES.shape_cols[p][o]) >> (4 * i)) & 0xFu;
                if (nib && ((nib + (nib & (~nib + 1u))) & nib)) return false;
            }
    return true;
}
static_assert(columns_contiguous(), "piece columns must be contiguous");

// Known answers from the reference tests (ta3_ai/tests/src/search/search_test.cpp:60-67).
static_assert(TABLES.nplace[0] == 17 && TABLES.nplace[1] == 9 && TABLES.nplace[2] == 34 && TABLES.nplace[3] == 17 &&
              TABLES.nplace[4] == 17 && TABLES.nplace[5] == 34 && TABLES.nplace[6] == 34, "placement counts");

// The kernel relies on the trees being perfect binary trees (node n of layer l
// has children 2n and 2n+1), which the hold rules produce for DEPTH = 4.
constexpr bool trees_are_binary() {
    for (int he = 0; he < 2; ++he)
        for (int l = 0; l < DEPTH; ++l) {
            if (TABLES.tree_count[he][l] != (2 << l)) return false;
            if (l + 1 < DEPTH)
                for (int n = 0; n < TABLES.tree_count[he][l]; ++n)
                    if (TABLES.tree[he][l][n].cbeg != 2 * n || TABLES.tree[he][l][n].cend != 2 * n + 2) return false;
        }
    return true;
}
static_assert(trees_are_binary(), "hold-plan trees must be perfect binary trees");

} // namespace ta3b
