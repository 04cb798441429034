// Candidate evaluation core, shared by the CUDA kernel and a host build used
// only by the CPU tests (tests/test_core_host.py) to pin the incremental path
// against the oracle before it runs on a GPU.
//
// A candidate = (parent board, placement). Two exact paths:
//
// * full path: the reference algorithm as written -- spawn-collision + drop
//   over the columns (ta3_sim/incl/ta3/sim/board2.hpp:306-320), lock
//   (board2.hpp:322-327), line clear (board2.hpp:333-342), the v11 features
//   recomputed over the whole board (ta3_ai/incl/ta3/ai/models/metrics/
//   v_board_metrics.hpp:130-232) and the 10 -> 8 -> 1 MLP
//   (ta3_ai/incl/ta3/ai/models/models/model_v11.hpp:63-91,166-180).
//
// * fast path: the same integers and floats, derived incrementally from a
//   per-parent record built once per kept frontier node. It applies when the
//   drop touches no cell in the piece's own rows of the spawn area (no
//   collision possible) and completes no row (no clear); otherwise the
//   candidate is handed to the full path. With no clear, the clear-count
//   inputs of the MLP are the parent's, so the first four multiply-adds of
//   every hidden unit are folded into the record (P[o]); the remaining
//   operations run in the reference order with separate roundings.
//
// Floating-point rules (both paths, host and device): every multiply and add
// rounds separately (__fmul_rn / __fadd_rn on the device; the host build uses
// -ffp-contract=off); sqrt is the correctly rounded sqrtf; divisions by the
// feature constants 20, 200, 5 and 100 use the FMA-corrected reciprocal
// quotient (Markstein), which tests/test_exact_division.py proves equal to
// the IEEE quotient over every value the features can take.
#pragma once
#include "tables.h"

#include <cstdint>
#if !defined(__CUDA_ARCH__)
#include <cmath>
#endif

#if defined(__CUDACC__)
#define TA3B_HD __host__ __device__ __forceinline__
#else
#define TA3B_HD inline
#endif

namespace ta3b {

// ------------------------------------------------------- exact arithmetic ---
TA3B_HD float f_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
TA3B_HD float f_add(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
TA3B_HD float f_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fmaf(a, b, c);
#endif
}
TA3B_HD float f_sqrt(float x) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(x);
#else
    return std::sqrt(x);
#endif
}
TA3B_HD int b_ctz_nz(uint32_t v) {           // v != 0
#if defined(__CUDA_ARCH__)
    return __ffs(int(v)) - 1;
#else
    return __builtin_ctz(v);
#endif
}
TA3B_HD int b_popc(uint32_t v) {
#if defined(__CUDA_ARCH__)
    return __popc(v);
#else
    return __builtin_popcount(v);
#endif
}
TA3B_HD int b_msb_nz(uint32_t v) {           // index of the highest set bit, v != 0
#if defined(__CUDA_ARCH__)
    return 31 - __clz(int(v));
#else
    return 31 - __builtin_clz(v);
#endif
}

// x / d rounded to nearest (Markstein: q = x*r, e = fma(-q, d, x), q' = fma(e, r, q)),
// exact for the feature domains (holes <= 230, hole depths <= 2599, wells <= 10,
// sqrt(surface sum) for sums <= 4761).
TA3B_HD float div_exact(float x, float d, float r) {
    float const q = f_mul(x, r);
    float const e = f_fma(-q, d, x);
    return f_fma(e, r, q);
}
constexpr float R20 = 0.05f, R200 = 0.005f, R5 = 0.2f, R100 = 0.01f;

TA3B_HD uint32_t ordered_bits(float v) {                         // beam.hpp:204-207
    uint32_t u;
#if defined(__CUDA_ARCH__)
    u = __float_as_uint(v);
#else
    __builtin_memcpy(&u, &v, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

TA3B_HD uint32_t clear_bump(int cleared) {                       // model_defs.hpp:177-183
    return cleared == 0 ? 0u : 1u << (8 * (cleared - 1));
}

TA3B_HD int column_top(uint32_t col) { return b_ctz_nz(col | FLOOR); }

// ------------------------------------------------------------ the weights ---
// Flat v11 layout (model_v11.hpp:166-180, utility.hpp:30-46): W1[o][i] at o*10+i,
// b1[o] at 80+o, W2[0][i] at 88+i, b2 at 96.
constexpr int WB1 = NIN * NHID, WW2 = WB1 + NHID, WB2 = WW2 + NHID;

// ----------------------------------------------------------- full path ---
// v_board_metrics.hpp:130-225 integer metrics of one board
struct BoardInts {
    uint32_t holes, hole_depths, max_height, wells;
    int surf_sq;
};

TA3B_HD int col_hole_depth(uint32_t col) {
    // occupied cells' count of empty cells below them: (H-1)n + n(n+1)/2 - (s + n^2),
    // s = sum of occupied row indices, taken from the 5 bit planes of the index
    int const n = b_popc(col);
    int const s = b_popc(col & 0x2AAAAAu) + 2 * b_popc(col & 0x4CCCCCu) + 4 * b_popc(col & 0x70F0F0u) +
                  8 * b_popc(col & 0x00FF00u) + 16 * b_popc(col & 0x7F0000u);
    return (H - 1) * n + n * (n + 1) / 2 - (s + n * n);
}

TA3B_HD BoardInts board_ints(uint32_t const (&b)[W]) {
    BoardInts r{0, 0, 0, 0, 0};
    int h[W];
#pragma unroll
    for (int x = 0; x < W; ++x) {
        h[x] = H - column_top(b[x]);
        r.holes += uint32_t(h[x] - b_popc(b[x]));
        r.max_height = uint32_t(h[x]) > r.max_height ? uint32_t(h[x]) : r.max_height;
        r.hole_depths += uint32_t(col_hole_depth(b[x]));
    }
#pragma unroll
    for (int x = 1; x < W; ++x) r.surf_sq += (h[x] - h[x - 1]) * (h[x] - h[x - 1]);
    uint32_t wells = uint32_t(h[1] >= h[0] + 3) + uint32_t(h[W - 2] >= h[W - 1] + 3);
#pragma unroll
    for (int x = 1; x < W - 1; ++x) wells += uint32_t(h[x - 1] >= h[x] + 3 && h[x + 1] >= h[x] + 3);
    r.wells = wells;
    return r;
}

// search.hpp:61-70: returns legality; nb = resulting board, cleared = rows removed
TA3B_HD bool apply_full(uint32_t const (&b)[W], uint32_t cols, int col0, uint32_t (&nb)[W], int& cleared) {
    uint32_t hit = 0;
    int drop = H;
    uint32_t nib[W];
#pragma unroll
    for (int x = 0; x < W; ++x) {
        uint32_t const d = uint32_t(x - col0);
        nib[x] = d < 4u ? (cols >> (4u * d)) & 0xFu : 0u;
        hit |= b[x] & nib[x];
        int const low = b_msb_nz(nib[x] | 1u);
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
    cleared = b_popc(full);
    if (full) {
#pragma unroll
        for (int x = 0; x < W; ++x) {
            uint32_t col = nb[x], fl = full;
            while (fl) {
                uint32_t const row = fl & (~fl + 1u);
                col = ((col & (row - 1u)) << 1) | (col & ~((row << 1) - 1u));
                fl ^= row;
            }
            nb[x] = col;
        }
    }
    return true;
}

// model_v11.hpp:63-91 inputs + forward, every operation in the reference order
template <class WF>
TA3B_HD float value_full(uint32_t clear_bits, BoardInts const& bi, bool held_i, WF const& w) {
    float in[NIN];
#pragma unroll
    for (int k = 0; k < 4; ++k) in[k] = f_mul(float((clear_bits >> (8 * k)) & 0xFFu), 0.25f);
    in[4] = div_exact(bi.surf_sq > 0 ? f_sqrt(float(bi.surf_sq)) : 0.0f, 100.0f, R100);
    in[5] = div_exact(float(bi.holes), 20.0f, R20);
    in[6] = div_exact(float(bi.hole_depths), 200.0f, R200);
    in[7] = float(bi.max_height);
    in[8] = held_i ? 1.0f : 0.0f;
    in[9] = div_exact(float(bi.wells), 5.0f, R5);
    float hid[NHID];
#pragma unroll
    for (int o = 0; o < NHID; ++o) {
        float v = w(WB1 + o);
#pragma unroll
        for (int i = 0; i < NIN; ++i) v = f_add(v, f_mul(in[i], w(o * NIN + i)));
        hid[o] = v > 0.0f ? v : 0.0f;                  // std::max<float>(0, v)
    }
    float v = w(WB2);
#pragma unroll
    for (int i = 0; i < NHID; ++i) v = f_add(v, f_mul(hid[i], w(WW2 + i)));
    return v;
}

// ---------------------------------------------- widened value network ---
// The reference's dense layers (ta3_ai/incl/ta3/ai/models/models/utility.hpp:29-46)
// widened: the v11 inputs -> H ReLU -> H ReLU -> 1 for a compile-time width H, per
// layer [out][in] weights then [out] biases (H = 64: 704 + 4160 + 65 = 4,929 parameters).
template <int H>
struct WideNet {
    static constexpr int B1 = NIN * H, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H, N = B3 + 1;
    // Device copy (STRIDE floats, 16-byte aligned): the same offsets, but layers 1 and 2
    // transposed to [in][out], so one input's weights to all H units are contiguous; the
    // word after the last bias is SKIP (the zero-term flag).
    static constexpr int W1T = 0, W2T = W2, SKIP = N, STRIDE = (N + 1 + 3) / 4 * 4;
    static_assert(H % 4 == 0 && B1 % 4 == 0 && W2 % 4 == 0 && B2 % 4 == 0 && W3 % 4 == 0 && STRIDE > SKIP,
                  "16-byte aligned blocks");
    // device-layout index of parameter j (reference order)
    static TA3B_HD int device_index(int j) {
        if (j < B1) return W1T + (j % NIN) * H + j / NIN;
        if (j >= W2 && j < B2) return W2T + ((j - W2) % H) * H + (j - W2) / H;
        return j;
    }
    static TA3B_HD bool is_bias(int j) { return (j >= B1 && j < W2) || (j >= B2 && j < W3) || j == B3; }
};
// the widths the kernels are built for: 64 (4,929 parameters, the 80k-sim widened generation) and 32 (1,441)
constexpr int WH = 64;
using Wide64 = WideNet<64>;
using Wide32 = WideNet<32>;
constexpr int NPARAMS_WIDE = Wide64::N, NPARAMS_WIDE32 = Wide32::N;
static_assert(NPARAMS_WIDE == 4929 && NPARAMS_WIDE32 == 1441 && Wide64::STRIDE == 4932, "10 -> H -> H -> 1");

TA3B_HD float relu(float v) { return v > 0.0f ? v : 0.0f; }    // std::max<float>(0, v)

// model_v11.hpp:63-91 inputs of the widened network
TA3B_HD void wide_inputs(uint32_t clear_bits, BoardInts const& bi, bool held_i, float (&in)[NIN]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) in[k] = f_mul(float((clear_bits >> (8 * k)) & 0xFFu), 0.25f);
    in[4] = div_exact(bi.surf_sq > 0 ? f_sqrt(float(bi.surf_sq)) : 0.0f, 100.0f, R100);
    in[5] = div_exact(float(bi.holes), 20.0f, R20);
    in[6] = div_exact(float(bi.hole_depths), 200.0f, R200);
    in[7] = float(bi.max_height);
    in[8] = held_i ? 1.0f : 0.0f;
    in[9] = div_exact(float(bi.wells), 5.0f, R5);
}

// --------------------------------------------------------- packed FP32x2 ---
// Two independent, separately rounded FP32 operations per instruction on
// sm_100 (__fmul2_rn / __fadd2_rn / __ffma2_rn: per component identical to the
// scalar _rn intrinsics). The host build applies the scalar operation twice.
#if !defined(__CUDACC__)
struct float2 {
    float x, y;
};
inline float2 make_float2(float x, float y) { return float2{x, y}; }
#endif
TA3B_HD float2 f2_mul(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __fmul2_rn(a, b);
#else
    return make_float2(f_mul(a.x, b.x), f_mul(a.y, b.y));
#endif
}
TA3B_HD float2 f2_add(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __fadd2_rn(a, b);
#else
    return make_float2(f_add(a.x, b.x), f_add(a.y, b.y));
#endif
}
TA3B_HD float2 f2_fma(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__)
    return __ffma2_rn(a, b, c);
#else
    return make_float2(f_fma(a.x, b.x, c.x), f_fma(a.y, b.y, c.y));
#endif
}
// The same two operations as inline PTX with the explicit .rn modifier, which
// PTX guarantees is never contracted into a fused multiply-add.
TA3B_HD float2 p2_mul(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long ua, ub, ud;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ua) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(ub) : "f"(b.x), "f"(b.y));
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(ud) : "l"(ua), "l"(ub));
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(ud));
    return d;
#else
    return make_float2(f_mul(a.x, b.x), f_mul(a.y, b.y));
#endif
}
TA3B_HD float2 p2_add(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long ua, ub, ud;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ua) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(ub) : "f"(b.x), "f"(b.y));
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(ud) : "l"(ua), "l"(ub));
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(ud));
    return d;
#else
    return make_float2(f_add(a.x, b.x), f_add(a.y, b.y));
#endif
}

// two correctly rounded quotients x / d (div_exact per component)
TA3B_HD float2 div2_exact(float2 x, float2 d, float2 r) {
    float2 const q = f2_mul(x, r);
    float2 const e = f2_fma(make_float2(-q.x, -q.y), d, x);
    return f2_fma(e, r, q);
}
TA3B_HD int dot4_s8(uint32_t a, uint32_t b) {                   // sum of 4 signed byte products
#if defined(__CUDA_ARCH__)
    return __dp4a(int(a), int(b), 0);
#else
    int s = 0;
    for (int i = 0; i < 4; ++i) s += int(int8_t(a >> (8 * i))) * int(int8_t(b >> (8 * i)));
    return s;
#endif
}

// ------------------------------------------------------ parent record ---
// One kept frontier node (or the committed board), in 68 u32 words (a 16-byte
// multiple; 68 = 4 mod 32 staggers the records across shared-memory banks):
constexpr int REC_WORDS = 68;
constexpr int R_P = 0;        // float[8]: hidden partial sums after the 4 clear inputs
constexpr int R_BOARD = 8;    // 10 bit-columns
constexpr int R_CLEARS = 18;  // path clear histogram (4 x 8-bit lanes)
constexpr int R_TOT = 19;     // holes (8) | max height (5) << 8 | wells (4) << 13 | surface sum (13) << 17
constexpr int R_HD = 20;      // hole depths total
constexpr int R_RC = 21;      // 3 words: occupied cells per row, 4 bits per row, rows 0..22
constexpr int R_HB = 24;      // 4 words: column heights as bytes (byte x = column x, bytes 10..15 zero)
constexpr int R_HMB = 28;     // 4 words: (holes - height) per column as signed bytes (bytes 10..15 zero)
constexpr int R_COMBO = 32;   // 34 words, per (c0, width) combo: the old surface terms of the window's pairs (12)
                              // | old wells of the window's columns (3) << 12 | left-well precondition << 15
                              // | height of column c0-1 (5) << 16 | right-well precondition << 21
                              // | height of column c0+w (5) << 22
static_assert(R_COMBO + NCOMBO <= REC_WORDS && REC_WORDS % 4 == 0, "record layout");
constexpr uint32_t WALL = 31; // height outside the board: satisfies every well-edge rule

// Column data a record is derived from: heights with walls (h[x + 2] = column x),
// holes per column, prefix sums of pair terms (pp[x+1] = sum over pairs (t-1, t),
// t <= x) and of well flags (pw[x+1] = wells among columns <= x).
struct ColumnData {
    int h[W + 4];
    int ho[W];
    int pp[W + 1], pw[W + 1];
    uint32_t holes, hd, maxh;
};

TA3B_HD void column_data(uint32_t const (&b)[W], ColumnData& c) {
    c.holes = c.hd = c.maxh = 0;
    c.h[0] = c.h[1] = c.h[W + 2] = c.h[W + 3] = int(WALL);
#pragma unroll
    for (int x = 0; x < W; ++x) {
        int const hx = H - column_top(b[x]);
        c.h[x + 2] = hx;
        c.ho[x] = hx - b_popc(b[x]);
        c.holes += uint32_t(c.ho[x]);
        c.maxh = uint32_t(hx) > c.maxh ? uint32_t(hx) : c.maxh;
    }
    c.pp[0] = c.pp[1] = c.pw[0] = 0;
#pragma unroll
    for (int x = 0; x < W; ++x) {
        int const l = c.h[x + 1], m = c.h[x + 2], r = c.h[x + 3];
        c.pw[x + 1] = c.pw[x] + int((l < r ? l : r) >= m + 3);
        if (x > 0) c.pp[x + 1] = c.pp[x] + (m - l) * (m - l);
    }
}

TA3B_HD uint32_t hole_depths_total(uint32_t const (&b)[W]) {
    uint32_t hd = 0;
#pragma unroll
    for (int x = 0; x < W; ++x) hd += uint32_t(col_hole_depth(b[x]));
    return hd;
}

TA3B_HD uint32_t row_counts(uint32_t const (&b)[W], int q) {
    // occupied cells per row, 4 bits per row, rows 8q..8q+7; summed bit-sliced
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
    for (int x = 0; x < W; ++x) {
        uint32_t const c0 = s0 & b[x];
        s0 ^= b[x];
        uint32_t const c1 = s1 & c0;
        s1 ^= c0;
        uint32_t const c2 = s2 & c1;
        s2 ^= c1;
        s3 ^= c2;
    }
    auto spread = [](uint32_t v) {              // 8 bits -> bit 4t of a word
        v &= 0xFFu;
        v = (v | (v << 12)) & 0x000F000Fu;
        v = (v | (v << 6)) & 0x03030303u;
        v = (v | (v << 3)) & 0x11111111u;
        return v;
    };
    return spread(s0 >> (8 * q)) | (spread(s1 >> (8 * q)) << 1) | (spread(s2 >> (8 * q)) << 2) |
           (spread(s3 >> (8 * q)) << 3);
}

// the byte arrays R_HB / R_HMB of a record
TA3B_HD void span_bytes(ColumnData const& c, uint32_t (&hb)[4], uint32_t (&hmb)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) hb[q] = hmb[q] = 0;
#pragma unroll
    for (int x = 0; x < W; ++x) {
        hb[x >> 2] |= uint32_t(c.h[x + 2]) << (8 * (x & 3));
        hmb[x >> 2] |= (uint32_t(c.ho[x] - c.h[x + 2]) & 0xFFu) << (8 * (x & 3));
    }
}

TA3B_HD uint32_t fshr32(uint32_t lo, uint32_t hi, uint32_t sh) {     // low word of (hi:lo) >> sh, sh < 32
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(lo, hi, sh);
#else
    return sh ? (lo >> sh) | (hi << (32u - sh)) : lo;
#endif
}

// window words for origin c0: bytes i = column c0+i (0 past the edge) of the two byte arrays
TA3B_HD void span_of(uint32_t const* rec, int c0, uint32_t& h4, uint32_t& hm4) {
    uint32_t const wi = uint32_t(c0) >> 2, sh = (uint32_t(c0) & 3u) * 8u;
    h4 = fshr32(rec[R_HB + wi], rec[R_HB + wi + 1], sh);
    hm4 = fshr32(rec[R_HMB + wi], rec[R_HMB + wi + 1], sh);
}

TA3B_HD uint32_t combo_word(ColumnData const& c, int c0, int wd) {
    int const last = c0 + wd < W - 1 ? c0 + wd : W - 1;                // window columns [c0-1, c0+w] in the board
    int const pairs = c.pp[last + 1] - c.pp[c0 > 1 ? c0 : 1];
    int const wells = c.pw[last + 1] - c.pw[c0 > 0 ? c0 - 1 : 0];
    uint32_t v = uint32_t(pairs) | (uint32_t(wells) << 12);
    if (c0 > 0) {
        int const hl = c.h[c0 + 1];                                     // column c0-1
        v |= (uint32_t(c.h[c0] >= hl + 3) << 15) | (uint32_t(hl) << 16);
    }
    if (c0 + wd < W) {
        int const hr = c.h[c0 + wd + 2];                                // column c0+w
        v |= (uint32_t(c.h[c0 + wd + 3] >= hr + 3) << 21) | (uint32_t(hr) << 22);
    }
    return v;
}

TA3B_HD void combo_of(int id, int& c0, int& wd) {
    wd = id < 10 ? 1 : id < 19 ? 2 : id < 27 ? 3 : 4;
    c0 = id - (wd == 1 ? 0 : wd == 2 ? 10 : wd == 3 ? 19 : 27);
}

template <class WF>
TA3B_HD uint32_t partial_word(uint32_t clear_bits, int o, WF const& w) {
    // hidden unit o through the 4 clear-count inputs (bias first, inputs ascending)
    float v = w(WB1 + o);
#pragma unroll
    for (int i = 0; i < 4; ++i) v = f_add(v, f_mul(f_mul(float((clear_bits >> (8 * i)) & 0xFFu), 0.25f), w(o * NIN + i)));
    uint32_t u;
#if defined(__CUDA_ARCH__)
    u = __float_as_uint(v);
#else
    __builtin_memcpy(&u, &v, 4);
#endif
    return u;
}

// PARTIALS: the v11 hidden partial sums (the widened network recomputes its own per candidate)
template <class WF, bool PARTIALS = true>
TA3B_HD void build_record(uint32_t const (&b)[W], uint32_t clear_bits, WF const& w, uint32_t* rec) {
    ColumnData c;
    column_data(b, c);
#pragma unroll
    for (int x = 0; x < W; ++x) rec[R_BOARD + x] = b[x];
    rec[R_CLEARS] = clear_bits;
    rec[R_TOT] = c.holes | (c.maxh << 8) | (uint32_t(c.pw[W]) << 13) | (uint32_t(c.pp[W]) << 17);
    rec[R_HD] = hole_depths_total(b);
#pragma unroll
    for (int q = 0; q < 3; ++q) rec[R_RC + q] = row_counts(b, q);
    // fully unrolled: every column index is a constant, so the column data stays in registers
    uint32_t hb[4], hmb[4];
    span_bytes(c, hb, hmb);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        rec[R_HB + q] = hb[q];
        rec[R_HMB + q] = hmb[q];
    }
#pragma unroll
    for (int id = 0; id < NCOMBO; ++id) {
        int c0, wd;
        combo_of(id, c0, wd);
        rec[R_COMBO + id] = combo_word(c, c0, wd);
    }
    if (PARTIALS) {
#pragma unroll
        for (int o = 0; o < NHID; ++o) rec[R_P + o] = partial_word(clear_bits, o, w);
    }
}

// ------------------------------------------------------------ fast path ---
// The weights the fast path needs, as pairs of hidden units (2q, 2q+1):
// W1[o][4..9], W2[o], plus b2.
struct FastW {
    float2 w4[NHID / 2], w5[NHID / 2], w6[NHID / 2], w7[NHID / 2], w8[NHID / 2], w9[NHID / 2], u[NHID / 2];
    float b2;
};

template <class WF>
TA3B_HD void load_fast_weights(WF const& w, FastW& f) {
#pragma unroll
    for (int q = 0; q < NHID / 2; ++q) {
        int const a = 2 * q, b = 2 * q + 1;
        f.w4[q] = make_float2(w(a * NIN + 4), w(b * NIN + 4));
        f.w5[q] = make_float2(w(a * NIN + 5), w(b * NIN + 5));
        f.w6[q] = make_float2(w(a * NIN + 6), w(b * NIN + 6));
        f.w7[q] = make_float2(w(a * NIN + 7), w(b * NIN + 7));
        f.w8[q] = make_float2(w(a * NIN + 8), w(b * NIN + 8));
        f.w9[q] = make_float2(w(a * NIN + 9), w(b * NIN + 9));
        f.u[q] = make_float2(w(WW2 + a), w(WW2 + b));
    }
    f.b2 = w(WB2);
}

enum FastStatus { FAST_OK = 0, FAST_DEFER = 1 };

// The parent record words a fast candidate reads.
struct RecView {
    float P[NHID];
    uint32_t tot, hd, rc0, rc1, rc2;
    uint32_t h4, hm4, combo;
};

// The placement's effect on the parent, from the record alone (branch-free).
// Returns FAST_DEFER when a piece cell may meet the stack inside the spawn rows
// or a row completes; the value is then meaningless.
// MLP arithmetic: MLP_SCALAR = __fmul_rn / __fadd_rn per hidden unit;
// MLP_PTX_X2 = pairs of hidden units per packed PTX instruction (mul/add.rn.f32x2);
// MLP_X2 = the same pairs through the __fmul2_rn / __fadd2_rn intrinsics;
// MLP_X2MUL = packed multiplies (__fmul2_rn), scalar adds. Each packed instruction rounds both
// halves exactly like the scalar .rn operation, but a packed multiply feeding a packed add is
// compiled into a fused multiply-add (one rounding): on the B200 the PTX pair equals fma.rn on
// all of 1,048,576 probe samples. Only MLP_X2MUL keeps the reference's two roundings.
enum MlpMode { MLP_SCALAR = 0, MLP_PTX_X2 = 1, MLP_X2 = 2, MLP_X2MUL = 3 };

// The fast path's features of one placement (holes, hole depths, surface,
// wells, max height) from the parent record alone; true when the candidate
// must take the full path instead.
struct FastFeat {
    int holes, hd, surf, wells, maxh, dr;
};

TA3B_HD bool fast_features(RecView const& r, PlaceFast pf, FastFeat& f) {
    int const width = int((pf.s >> 22) & 7u);
    // drop = min over the piece's columns of (top - lowest piece cell - 1), top = H - height
    int drop = 255, sumd = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int const d = int((pf.d4 >> (8 * i)) & 0xFFu) - int((r.h4 >> (8 * i)) & 0xFFu);
        drop = d < drop ? d : drop;
        sumd += i < width ? d : 0;
    }
    bool defer = drop < 0;
    int const dr = defer ? 0 : drop;
    // rows dr..dr+3: occupied cells + the piece's cells per row; a nibble of 10 = a full row
    int const bit = 4 * dr;
    uint32_t const wlo = bit < 32 ? r.rc0 : (bit < 64 ? r.rc1 : r.rc2);
    uint32_t const whi = bit < 32 ? r.rc1 : (bit < 64 ? r.rc2 : 0u);
    uint32_t const sh = uint32_t(bit & 31);
    uint32_t const win = (sh ? ((wlo >> sh) | (whi << (32u - sh))) : wlo) & 0xFFFFu;
    uint32_t const sum = (win + (pf.m & 0xFFFFu)) ^ 0xAAAAu;
    defer = defer || (((sum - 0x1111u) & ~sum & 0x8888u) != 0u);
    // holes gain the gaps under the piece; every new cell sits over (holes + gap) empty cells
    int const holes = int(r.tot & 0xFFu) + sumd - width * dr;
    int const hd = int(r.hd) + dot4_s8(pf.c4, r.hm4) + int((pf.s >> 7) & 0x7Fu) - 4 * dr;
    int const top_max = H - dr - int((pf.m >> 25) & 3u);
    int const maxh = int((r.tot >> 8) & 0x1Fu) > top_max ? int((r.tot >> 8) & 0x1Fu) : top_max;
    int const n0 = H - dr - int((pf.s >> 18) & 3u);              // new height of the first / last piece column
    int const nl = H - dr - int((pf.s >> 20) & 3u);
    uint32_t const cb = r.combo;
    int const hl = int((cb >> 16) & 31u), hr = int((cb >> 22) & 31u);
    bool const lv = (pf.m >> 23) & 1u, rv = (pf.m >> 24) & 1u;
    // surface: the window's pairs are replaced by the piece's inner steps and the two edge pairs
    int surf = int(r.tot >> 17) - int(cb & 0xFFFu) + int((pf.s >> 14) & 0xFu);
    surf += lv ? (n0 - hl) * (n0 - hl) : 0;
    surf += rv ? (hr - nl) * (hr - nl) : 0;
    // wells: only the two neighbour columns (and a one-column piece itself) can be wells now
    int wells = int((r.tot >> 13) & 0xFu) - int((cb >> 12) & 7u);
    wells += int(lv && ((cb >> 15) & 1u) && n0 >= hl + 3);
    wells += int(rv && ((cb >> 21) & 1u) && nl >= hr + 3);
    int const hlw = lv ? hl : int(WALL), hrw = rv ? hr : int(WALL);
    wells += int(((pf.m >> 22) & 1u) && (hlw < hrw ? hlw : hrw) >= n0 + 3);
    f = FastFeat{holes, hd, surf, wells, maxh, dr};
    return defer;
}

template <int MLP = MLP_SCALAR>
TA3B_HD int fast_eval(RecView const& r, PlaceFast pf, bool held_i, FastW const& fw, float& value,
                      float* dbg = nullptr) {
    FastFeat ff;
    bool const defer = fast_features(r, pf, ff);
    int const holes = ff.holes, hd = ff.hd, surf = ff.surf, wells = ff.wells, maxh = ff.maxh, dr = ff.dr;
    // features (model_v11.hpp:63-91): pairs of correctly rounded quotients
    float const sq = surf > 0 ? f_sqrt(float(surf)) : 0.0f;
    float2 const q56 = div2_exact(make_float2(float(holes), float(hd)), make_float2(20.0f, 200.0f),
                                  make_float2(R20, R200));
    float2 const q94 = div2_exact(make_float2(float(wells), sq), make_float2(5.0f, 100.0f), make_float2(R5, R100));
    float2 const x4 = make_float2(q94.y, q94.y), x5 = make_float2(q56.x, q56.x), x6 = make_float2(q56.y, q56.y);
    float const m7 = float(maxh), m8 = held_i ? 1.0f : 0.0f;
    float2 const x7 = make_float2(m7, m7), x8 = make_float2(m8, m8), x9 = make_float2(q94.x, q94.x);
    if (dbg) {                                   // diagnostics for the self-tests
        dbg[0] = float(holes); dbg[1] = float(hd); dbg[2] = float(surf); dbg[3] = float(wells);
        dbg[4] = float(maxh); dbg[5] = x4.x; dbg[6] = x5.x; dbg[7] = x6.x; dbg[8] = x9.x; dbg[9] = float(dr);
    }
    // hidden units in pairs, every multiply and add rounded separately, reference order
    float v = fw.b2;
#pragma unroll
    for (int q = 0; q < NHID / 2; ++q) {
        float2 a = make_float2(r.P[2 * q], r.P[2 * q + 1]);
        if (MLP == MLP_X2MUL) {
            float2 const m4 = f2_mul(x4, fw.w4[q]), m5 = f2_mul(x5, fw.w5[q]), m6 = f2_mul(x6, fw.w6[q]);
            float2 const m7 = f2_mul(x7, fw.w7[q]), m8 = f2_mul(x8, fw.w8[q]), m9 = f2_mul(x9, fw.w9[q]);
            a.x = f_add(a.x, m4.x);
            a.y = f_add(a.y, m4.y);
            a.x = f_add(a.x, m5.x);
            a.y = f_add(a.y, m5.y);
            a.x = f_add(a.x, m6.x);
            a.y = f_add(a.y, m6.y);
            a.x = f_add(a.x, m7.x);
            a.y = f_add(a.y, m7.y);
            a.x = f_add(a.x, m8.x);
            a.y = f_add(a.y, m8.y);
            a.x = f_add(a.x, m9.x);
            a.y = f_add(a.y, m9.y);
        } else if (MLP == MLP_X2) {
            a = f2_add(a, f2_mul(x4, fw.w4[q]));
            a = f2_add(a, f2_mul(x5, fw.w5[q]));
            a = f2_add(a, f2_mul(x6, fw.w6[q]));
            a = f2_add(a, f2_mul(x7, fw.w7[q]));
            a = f2_add(a, f2_mul(x8, fw.w8[q]));
            a = f2_add(a, f2_mul(x9, fw.w9[q]));
        } else if (MLP == MLP_PTX_X2) {
            a = p2_add(a, p2_mul(x4, fw.w4[q]));
            a = p2_add(a, p2_mul(x5, fw.w5[q]));
            a = p2_add(a, p2_mul(x6, fw.w6[q]));
            a = p2_add(a, p2_mul(x7, fw.w7[q]));
            a = p2_add(a, p2_mul(x8, fw.w8[q]));
            a = p2_add(a, p2_mul(x9, fw.w9[q]));
        } else {
            a.x = f_add(a.x, f_mul(x4.x, fw.w4[q].x));
            a.y = f_add(a.y, f_mul(x4.y, fw.w4[q].y));
            a.x = f_add(a.x, f_mul(x5.x, fw.w5[q].x));
            a.y = f_add(a.y, f_mul(x5.y, fw.w5[q].y));
            a.x = f_add(a.x, f_mul(x6.x, fw.w6[q].x));
            a.y = f_add(a.y, f_mul(x6.y, fw.w6[q].y));
            a.x = f_add(a.x, f_mul(x7.x, fw.w7[q].x));
            a.y = f_add(a.y, f_mul(x7.y, fw.w7[q].y));
            a.x = f_add(a.x, f_mul(x8.x, fw.w8[q].x));
            a.y = f_add(a.y, f_mul(x8.y, fw.w8[q].y));
            a.x = f_add(a.x, f_mul(x9.x, fw.w9[q].x));
            a.y = f_add(a.y, f_mul(x9.y, fw.w9[q].y));
        }
        if (dbg) {
            dbg[10 + 2 * q] = a.x;
            dbg[11 + 2 * q] = a.y;
        }
        a.x = a.x > 0.0f ? a.x : 0.0f;                      // std::max<float>(0, v)
        a.y = a.y > 0.0f ? a.y : 0.0f;
        float2 const t = MLP == MLP_PTX_X2                  ? p2_mul(a, fw.u[q])
                         : (MLP == MLP_X2 || MLP == MLP_X2MUL) ? f2_mul(a, fw.u[q])
                                                               : make_float2(f_mul(a.x, fw.u[q].x),
                                                                             f_mul(a.y, fw.u[q].y));
        v = f_add(v, t.x);
        v = f_add(v, t.y);
    }
    value = v;
    return defer ? FAST_DEFER : FAST_OK;
}

// The fast path's inputs of the widened network: the same features, the parent's
// clear counts as the first four inputs (a fast candidate clears no row). Returns
// true when the candidate must take the full path instead (inputs then all zero).
TA3B_HD bool fast_wide_inputs(RecView const& r, uint32_t clear_bits, PlaceFast pf, bool held_i, float (&in)[NIN]) {
    FastFeat ff;
    bool const defer = fast_features(r, pf, ff);
    BoardInts bi;
    bi.surf_sq = ff.surf;
    bi.holes = ff.holes;
    bi.hole_depths = ff.hd;
    bi.max_height = ff.maxh;
    bi.wells = ff.wells;
    wide_inputs(clear_bits, bi, held_i, in);
    if (defer)
#pragma unroll
        for (int i = 0; i < NIN; ++i) in[i] = 0.0f;
    return defer;
}

} // namespace ta3b
