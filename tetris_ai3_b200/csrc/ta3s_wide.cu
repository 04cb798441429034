// Surrogate fitness model for any parameter-vector size: an MLP in -> H -> H -> 2
// (predicted mean score, log-variance), the v11 surrogate's scheme scaled to the
// widened evaluator (in = 4,929 parameters, H = 256). No counterpart in the
// reference; the C ABI is the ta3w_* part of include/ta3b_surrogate.h.
//
// Layer by layer instead of one fused kernel (the first layer's weights alone are
// H x in = 1.3 M values): every matrix product is one launch of gemm_kernel, a
// tcgen05.mma (kind::f16, BF16 operands staged in shared memory, FP32
// accumulators in tensor memory) GEMM on 128 x 128 output tiles with K in
// stages of 64 and optional split-K; the bias, ReLU, output layer, loss and
// bias gradients run in small CUDA-core kernels between them. Every reduction
// runs in a fixed order, so two identical calls give identical bits.
//
// Operand tiles (128 rows of M or N by 64 of K, BF16, no swizzle) are built from
// 8 x 8 core matrices of 128 contiguous bytes. An operand whose global rows run
// along K (K-major) stores element (r, k) at (r/8)*1024 + (k/8)*128 + (r%8)*16 +
// (k%8)*2 and is described with LBO 128 (next 8 K) and SBO 1024 (next 8 rows);
// an operand whose global rows run along M/N (MN-major: the weight-gradient
// products, where K is the batch) stores element (k, r) at (k/8)*2048 +
// (r/8)*128 + (k%8)*16 + (r%8)*2 with LBO 2048 (next 8 K) and SBO 128 (next 8
// of M/N). Either way one 16-byte global load fills one core-matrix row.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/ta3b_surrogate.h"

namespace ta3w {

constexpr int TILE = 128;                       // M and N per output tile
constexpr int KS = 64;                          // K per shared-memory stage
constexpr int THREADS = 128;
constexpr uint32_t OP_BYTES = TILE * KS * 2;    // one operand stage: 16 KB
constexpr uint32_t S_BAR = 4 * OP_BYTES;        // two stages of A and B, then two mbarriers
constexpr uint32_t S_TMEM = S_BAR + 16;
constexpr uint32_t SMEM_BYTES = S_TMEM + 16 + 1024;   // + alignment slack
constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL;  // ~2 s at 1.9 GHz

// tcgen05 shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}
// instruction descriptor: D F32, A/B BF16, majors (0 = K, 1 = MN), N = 128, M = 128
__host__ __device__ constexpr uint32_t instr_desc(int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           (uint32_t(TILE >> 3) << 17) | (uint32_t(TILE >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bounded wait for the completion of the barrier phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    long long const t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > WAIT_LIMIT_CYCLES) return false;
    }
}

// C[split][M][N] (FP32) = sum over this split's K of A(m, k) B(n, k), where
//   A(m, k) = A_MN ? a[k' * lda + m] : a[m' * lda + k]   (BF16; ' = through a_idx when given,
//   B(n, k) = B_MN ? b[k' * ldb + n] : b[n' * ldb + k]    a negative index reads zeros)
// M, N multiples of 128; K and k_split multiples of 64. Grid (M/128, N/128, splits).
struct GemmArgs {
    __nv_bfloat16 const* a;
    int64_t lda;
    int32_t const* a_idx;
    __nv_bfloat16 const* b;
    int64_t ldb;
    int32_t const* b_idx;
    float* c;
    int64_t ldc;
    int64_t c_split;       // floats between consecutive splits' outputs
    int m, n, k, k_split;
    uint32_t* status;      // bit 0: a tensor-core wait timed out
};

// one operand stage (128 rows of M/N x 64 of K) from global memory into its core-matrix layout
template <int MN>
__device__ __forceinline__ void stage_operand(uint8_t* dst, __nv_bfloat16 const* src, int64_t ld,
                                              int32_t const* idx, int r0, int k0, int tid) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        int const c = tid + THREADS * q;               // 1,024 16-byte chunks
        int outer, inner;
        uint32_t off;
        if (MN) {                                      // global rows = K, 16 chunks of 8 along M/N
            int const kr = c >> 4, j = c & 15;
            outer = k0 + kr;
            inner = r0 + 8 * j;
            off = uint32_t((kr >> 3) * 2048 + j * 128 + (kr & 7) * 16);
        } else {                                       // global rows = M/N, 8 chunks of 8 along K
            int const r = c >> 3, j = c & 7;
            outer = r0 + r;
            inner = k0 + 8 * j;
            off = uint32_t((r >> 3) * 1024 + j * 128 + (r & 7) * 16);
        }
        if (idx) outer = idx[outer];
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (outer >= 0) v = __ldg(reinterpret_cast<uint4 const*>(src + outer * ld + inner));
        *reinterpret_cast<uint4*>(dst + off) = v;
    }
}

template <int A_MN, int B_MN>
__global__ void __launch_bounds__(THREADS, 1) gemm_kernel(GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint32_t const sbase = uint32_t(__cvta_generic_to_shared(sm));
    int const tid = threadIdx.x, warp = tid >> 5;
    int const m0 = blockIdx.x * TILE, n0 = blockIdx.y * TILE;
    int const kb = blockIdx.z * g.k_split;
    int const ke = min(g.k, kb + g.k_split);
    int const nk = (ke - kb) / KS;
    uint32_t const bar0 = sbase + S_BAR;                // stage b's barrier: bar0 + 8 b
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + S_TMEM);
    volatile uint32_t* abort_s = reinterpret_cast<volatile uint32_t*>(sm + S_TMEM + 4);
    if (tid == 0) {
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        *abort_s = 0u;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + S_TMEM),
                     "r"(uint32_t(TILE)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    uint32_t const tmem = *tmem_slot;
    uint32_t const idesc = instr_desc(A_MN, B_MN);
    for (int it = 0; it < nk; ++it) {
        int const buf = it & 1;
        // the stage's buffers are free once the MMAs of two iterations ago completed
        if (tid == 0 && it >= 2 && !mbar_wait(bar0 + 8 * buf, uint32_t((it - 2) >> 1) & 1u)) {
            *abort_s = 1u;
            atomicOr(g.status, 1u);
        }
        __syncthreads();
        if (*abort_s) break;
        uint8_t* const as = sm + buf * 2 * OP_BYTES;
        uint8_t* const bs = as + OP_BYTES;
        int const k0 = kb + it * KS;
        stage_operand<A_MN>(as, g.a, g.lda, g.a_idx, m0, k0, tid);
        stage_operand<B_MN>(bs, g.b, g.ldb, g.b_idx, n0, k0, tid);
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (tid == 0) {
            uint32_t const a_s = sbase + buf * 2 * OP_BYTES, b_s = a_s + OP_BYTES;
#pragma unroll
            for (int kk = 0; kk < KS / 16; ++kk) {
                uint64_t const ad = A_MN ? smem_desc(a_s + kk * 4096, 2048, 128) : smem_desc(a_s + kk * 256, 128, 1024);
                uint64_t const bd = B_MN ? smem_desc(b_s + kk * 4096, 2048, 128) : smem_desc(b_s + kk * 256, 128, 1024);
                mma_bf16(tmem, ad, bd, idesc, (it > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(bar0 + 8 * buf);
        }
    }
    // the last commit completes after every MMA of this CTA
    if (tid == 0 && !*abort_s && nk > 0 && !mbar_wait(bar0 + 8 * ((nk - 1) & 1), uint32_t((nk - 1) >> 1) & 1u)) {
        *abort_s = 1u;
        atomicOr(g.status, 1u);
    }
    __syncthreads();
    fence_after();
    if (!*abort_s) {
        // TMEM lane t = output row m0 + t
        float* const crow = g.c + int64_t(blockIdx.z) * g.c_split + int64_t(m0 + tid) * g.ldc + n0;
        uint32_t const lane_base = tmem + (uint32_t(warp * 32) << 16);
        for (int cc = 0; cc < TILE / 16; ++cc) {
            float v[16];
            if (nk > 0) tmem_ld16(lane_base + cc * 16, v);
            else
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0.f;
#pragma unroll
            for (int j = 0; j < 16; j += 4)
                *reinterpret_cast<float4*>(crow + cc * 16 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(TILE)) : "memory");
}

using GemmFn = void (*)(GemmArgs);
GemmFn gemm_fn(int a_mn, int b_mn) {
    return a_mn ? (b_mn ? gemm_kernel<1, 1> : gemm_kernel<1, 0>) : (b_mn ? gemm_kernel<0, 1> : gemm_kernel<0, 0>);
}

// ---------------------------------------------------------- model kernels ---
struct Dims {
    int in, inp, h;          // input size, padded to a multiple of 128; hidden width (multiple of 128)
    int64_t w1, w2, w3, b1, b2, b3, n;   // parameter offsets (FP32 vector) and count
};
inline Dims make_dims(int in, int h) {
    Dims d;
    d.in = in;
    d.inp = (in + TILE - 1) / TILE * TILE;     // the N of dW1 = dH1^T X: a whole number of tiles
    d.h = h;
    d.w1 = 0;
    d.w2 = d.w1 + int64_t(h) * d.inp;
    d.w3 = d.w2 + int64_t(h) * h;
    d.b1 = d.w3 + 2 * int64_t(h);
    d.b2 = d.b1 + h;
    d.b3 = d.b2 + h;
    d.n = d.b3 + 2;
    return d;
}

// the pass's row map: out[r] = idx[r] (or r without idx) for r < valid, -1 (a zero row) after
__global__ void rowmap_kernel(int32_t const* __restrict__ idx, int valid, int rows, int32_t* __restrict__ out) {
    int const r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < rows) out[r] = r < valid ? (idx ? idx[r] : r) : -1;
}

// standardised FP32 rows [rows][in] -> BF16 [rows][inp] (padding columns zero)
__global__ void pack_kernel(float const* __restrict__ x, int rows, int in, int inp, float const* __restrict__ mean,
                            float const* __restrict__ inv_std, __nv_bfloat16* __restrict__ xb) {
    int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(rows) * inp) return;
    int64_t const r = i / inp;
    int const c = int(i % inp);
    float const v = c < in ? (x[r * in + c] - mean[c]) * inv_std[c] : 0.f;
    xb[i] = __float2bfloat16_rn(v);
}

// H1 = BF16(relu(sum of the split partials + b1)), [rows][h]
__global__ void act1_kernel(float const* __restrict__ part, int splits, int64_t split_stride, int rows, int h,
                            float const* __restrict__ b1, __nv_bfloat16* __restrict__ h1b) {
    int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= int64_t(rows) * h) return;
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += part[k * split_stride + i];
    s += b1[i % h];
    h1b[i] = __float2bfloat16_rn(s > 0.f ? s : 0.f);
}

// Output layer, loss and the first backward step, one thread per row:
//   z2 = F2 + b2, h2 = relu(z2), (mu, s) = W3 h2 + b3 (FP32, ascending);
//   training rows (y given, row valid): NLL 0.5 (s' + (y - mu)^2 e^-s'), s' = clamp(s, +-12),
//   dmu, ds of the batch mean, dH2 = BF16((z2 > 0) (dmu W3[0] + ds W3[1])).
__global__ void head_kernel(float const* __restrict__ f2, int rows, int valid_rows, int h,
                            float const* __restrict__ p, int64_t off_w3, int64_t off_b2, int64_t off_b3,
                            float const* __restrict__ y, int32_t const* __restrict__ idx, float inv_n,
                            float* __restrict__ out, float* __restrict__ h2f, float* __restrict__ gcols,
                            float* __restrict__ row_loss, __nv_bfloat16* __restrict__ dh2b) {
    int const r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float const* z = f2 + int64_t(r) * h;
    float const* w3 = p + off_w3;
    float const* b2 = p + off_b2;
    float o0 = p[off_b3], o1 = p[off_b3 + 1];
    for (int o = 0; o < h; ++o) {
        float const v = z[o] + b2[o];
        float const hv = v > 0.f ? v : 0.f;
        o0 = fmaf(hv, w3[o], o0);
        o1 = fmaf(hv, w3[h + o], o1);
        if (h2f) h2f[int64_t(r) * h + o] = hv;
    }
    if (out) {
        out[2 * r] = o0;
        out[2 * r + 1] = o1;
    }
    if (!y) return;
    int const src = r < valid_rows ? (idx ? idx[r] : r) : -1;
    float dmu = 0.f, ds = 0.f, loss = 0.f;
    if (src >= 0) {
        float const s = fminf(fmaxf(o1, -12.f), 12.f);
        float const e = expf(-s);
        float const d = y[src] - o0;
        loss = 0.5f * (s + d * d * e);
        dmu = -d * e * inv_n;
        ds = (o1 > -12.f && o1 < 12.f) ? 0.5f * (1.f - d * d * e) * inv_n : 0.f;
    }
    gcols[2 * r] = dmu;
    gcols[2 * r + 1] = ds;
    row_loss[r] = loss;
    for (int o = 0; o < h; ++o) {
        float const v = z[o] + b2[o];
        dh2b[int64_t(r) * h + o] = __float2bfloat16_rn(v > 0.f ? fmaf(dmu, w3[o], ds * w3[h + o]) : 0.f);
    }
}

// dH1 = BF16((H1 > 0) * F3), [rows][h]
__global__ void mask1_kernel(float const* __restrict__ f3, __nv_bfloat16 const* __restrict__ h1b, int64_t n,
                             __nv_bfloat16* __restrict__ dh1b) {
    int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dh1b[i] = __float2bfloat16_rn(__bfloat162float(h1b[i]) > 0.f ? f3[i] : 0.f);
}

// Column sums over the batch rows in order: db1, db2 (of the BF16 dH1, dH2),
// dW3 = sum h2 [dmu, ds], db3, and the summed loss. One thread per hidden unit.
__global__ void small_grads_kernel(int rows, int h, __nv_bfloat16 const* __restrict__ dh1b,
                                   __nv_bfloat16 const* __restrict__ dh2b, float const* __restrict__ h2f,
                                   float const* __restrict__ gcols, float const* __restrict__ row_loss,
                                   float* __restrict__ grad, int64_t off_w3, int64_t off_b1, int64_t off_b2,
                                   int64_t off_b3, float* __restrict__ loss_out) {
    int const o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < h) {
        float s1 = 0.f, s2 = 0.f, w0 = 0.f, w1 = 0.f;
        for (int r = 0; r < rows; ++r) {
            int64_t const i = int64_t(r) * h + o;
            s1 += __bfloat162float(dh1b[i]);
            s2 += __bfloat162float(dh2b[i]);
            w0 = fmaf(h2f[i], gcols[2 * r], w0);
            w1 = fmaf(h2f[i], gcols[2 * r + 1], w1);
        }
        grad[off_b1 + o] = s1;
        grad[off_b2 + o] = s2;
        grad[off_w3 + o] = w0;
        grad[off_w3 + h + o] = w1;
    } else if (o < h + 3) {
        int const c = o - h;        // 0, 1: db3; 2: loss
        float s = 0.f;
        for (int r = 0; r < rows; ++r) s += c < 2 ? gcols[2 * r + c] : row_loss[r];
        if (c < 2) grad[off_b3 + c] = s;
        else if (loss_out) *loss_out = s;
    }
}

// AdamW over the flat parameter vector (padding columns of W1 stay zero), then
// the BF16 copies of W1 and W2 the GEMMs read.
__global__ void adam_kernel(float* __restrict__ param, float* __restrict__ m, float* __restrict__ v,
                            float const* __restrict__ grad, int64_t n, int64_t off_w2, int64_t off_w3, int in,
                            int inp, float lr, float b1, float b2, float eps, float c1, float c2, float wd,
                            __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b) {
    int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i < off_w2 && int(i % inp) >= in) return;
    float const g = grad[i];
    float const mi = b1 * m[i] + (1.f - b1) * g;
    float const vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float const w = param[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps) - lr * wd * param[i];
    param[i] = w;
    if (i < off_w2) w1b[i] = __float2bfloat16_rn(w);
    else if (i < off_w3) w2b[i - off_w2] = __float2bfloat16_rn(w);
}

__global__ void refresh_kernel(float const* __restrict__ param, int64_t off_w2, int64_t off_w3,
                               __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b) {
    int64_t const i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < off_w2) w1b[i] = __float2bfloat16_rn(param[i]);
    else if (i < off_w3) w2b[i - off_w2] = __float2bfloat16_rn(param[i]);
}

} // namespace ta3w

using namespace ta3w;

struct ta3w_model {
    int device = 0;
    int sms = 0;
    Dims d{};
    std::string err;
    cudaStream_t stream = nullptr;
    float* d_param = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_grad = nullptr;
    __nv_bfloat16* d_w1b = nullptr;
    __nv_bfloat16* d_w2b = nullptr;
    uint32_t* d_status = nullptr;
    float* d_loss = nullptr;
    float* d_stats = nullptr;          // mean [inp], inv_std [inp]
    std::vector<float> x_mean, x_inv_std;
    float y_mean = 0.f, y_std = 1.f;
    // data
    uint32_t rows = 0;
    size_t cap_rows = 0;
    float* d_xraw = nullptr;
    __nv_bfloat16* d_x = nullptr;
    float* d_y = nullptr;
    int32_t* d_idx = nullptr;
    size_t cap_idx = 0;
    // activations for up to cap_act rows (a multiple of 128)
    size_t cap_act = 0;
    int max_splits = 1;
    float* d_f1 = nullptr;             // [splits][rows][h]
    __nv_bfloat16* d_h1b = nullptr;
    float* d_f2 = nullptr;             // F2, then F3
    float* d_h2f = nullptr;
    float* d_gcols = nullptr;
    float* d_rowloss = nullptr;
    __nv_bfloat16* d_dh2b = nullptr;
    __nv_bfloat16* d_dh1b = nullptr;
    float* d_out = nullptr;
    int32_t* d_rowidx = nullptr;       // identity / padded row map of a full pass
    uint64_t adam_t = 0;
};

namespace {
thread_local std::string g_werr;

#define TA3W_CUDA(m, call, what)                                                               \
    do {                                                                                       \
        cudaError_t const e_ = (call);                                                         \
        if (e_ != cudaSuccess) return wfail(m, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int wfail(ta3w_model* m, std::string msg) {
    if (m) m->err = msg;
    g_werr = msg;
    return 1;
}

template <class T>
int wgrow(ta3w_model* m, T*& ptr, size_t& cap, size_t n, char const* what) {
    if (n <= cap && ptr) return 0;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    TA3W_CUDA(m, cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)), what);
    cap = n;
    return 0;
}
template <class T>
int walloc(ta3w_model* m, T*& ptr, size_t n, char const* what) {
    size_t cap = 0;
    return wgrow(m, ptr, cap, n, what);
}

int round128(int n) { return (n + TILE - 1) / TILE * TILE; }
// rows of one forward / backward pass: bounds the activation buffers (split-K partials
// of the first layer alone take splits x rows x H floats)
constexpr uint32_t kMaxPassRows = 65536;

// activation buffers for `rows` (a multiple of 128) rows
int ensure_act(ta3w_model* m, size_t rows) {
    if (rows <= m->cap_act) return 0;
    int const h = m->d.h;
    int const splits = m->max_splits;
    for (void* p : {(void*)m->d_f1, (void*)m->d_h1b, (void*)m->d_f2, (void*)m->d_h2f, (void*)m->d_gcols,
                    (void*)m->d_rowloss, (void*)m->d_dh2b, (void*)m->d_dh1b, (void*)m->d_out, (void*)m->d_rowidx})
        if (p) cudaFree(p);
    m->d_f1 = m->d_f2 = m->d_h2f = m->d_gcols = m->d_rowloss = m->d_out = nullptr;
    m->d_h1b = m->d_dh2b = m->d_dh1b = nullptr;
    m->d_rowidx = nullptr;
    m->cap_act = 0;
    if (walloc(m, m->d_f1, size_t(splits) * rows * h, "alloc F1") || walloc(m, m->d_h1b, rows * h, "alloc H1") ||
        walloc(m, m->d_f2, rows * h, "alloc F2") || walloc(m, m->d_h2f, rows * h, "alloc H2") ||
        walloc(m, m->d_gcols, rows * 2, "alloc G") || walloc(m, m->d_rowloss, rows, "alloc loss rows") ||
        walloc(m, m->d_dh2b, rows * h, "alloc dH2") || walloc(m, m->d_dh1b, rows * h, "alloc dH1") ||
        walloc(m, m->d_out, rows * 2, "alloc outputs") || walloc(m, m->d_rowidx, rows, "alloc row map"))
        return 1;
    m->cap_act = rows;
    return 0;
}

int gemm(ta3w_model* m, int a_mn, int b_mn, __nv_bfloat16 const* a, int64_t lda, int32_t const* a_idx,
         __nv_bfloat16 const* b, int64_t ldb, int32_t const* b_idx, float* c, int64_t ldc, int64_t c_split, int M,
         int N, int K, int splits) {
    int const kst = K / KS;
    int const per = (kst + splits - 1) / splits;
    splits = (kst + per - 1) / per;
    GemmArgs g{a, lda, a_idx, b, ldb, b_idx, c, ldc, c_split, M, N, K, per * KS, m->d_status};
    gemm_fn(a_mn, b_mn)<<<dim3(M / TILE, N / TILE, splits), THREADS, SMEM_BYTES, m->stream>>>(g);
    TA3W_CUDA(m, cudaGetLastError(), "gemm launch");
    return 0;
}

int splits_for(ta3w_model* m, int M, int N, int K) {
    int const tiles = (M / TILE) * (N / TILE);
    int const want = std::max(1, (m->sms + tiles - 1) / tiles);
    return std::min({want, K / KS, m->max_splits});
}

// forward (and with y, the backward pass into d_grad) over `rows` rows of d_x
// selected by idx (device, `rows` entries, -1 = none; rows padded to 128 here)
int pass(ta3w_model* m, int32_t const* idx, int valid_rows, bool train) {
    Dims const& d = m->d;
    int const R = round128(valid_rows);
    if (ensure_act(m, size_t(R))) return 1;
    int const h = d.h;
    rowmap_kernel<<<unsigned((R + 255) / 256), 256, 0, m->stream>>>(idx, valid_rows, R, m->d_rowidx);
    TA3W_CUDA(m, cudaGetLastError(), "row map");
    int32_t const* rows = m->d_rowidx;
    // layer 1: F1 = X W1^T (M = rows, N = h, K = inp), split over K
    int const s1 = splits_for(m, R, h, d.inp);
    int64_t const f1_stride = int64_t(R) * h;
    if (gemm(m, 0, 0, m->d_x, d.inp, rows, m->d_w1b, d.inp, nullptr, m->d_f1, h, f1_stride, R, h, d.inp, s1)) return 1;
    int const per = (d.inp / KS + s1 - 1) / s1;
    int const s1_used = (d.inp / KS + per - 1) / per;
    int64_t const n_act = int64_t(R) * h;
    act1_kernel<<<unsigned((n_act + 255) / 256), 256, 0, m->stream>>>(m->d_f1, s1_used, f1_stride, R, h,
                                                                      m->d_param + d.b1, m->d_h1b);
    TA3W_CUDA(m, cudaGetLastError(), "act1");
    // layer 2: F2 = H1 W2^T
    if (gemm(m, 0, 0, m->d_h1b, h, nullptr, m->d_w2b, h, nullptr, m->d_f2, h, 0, R, h, h, 1)) return 1;
    head_kernel<<<unsigned((R + 127) / 128), 128, 0, m->stream>>>(
        m->d_f2, R, valid_rows, h, m->d_param, d.w3, d.b2, d.b3, train ? m->d_y : nullptr, rows,
        1.0f / float(valid_rows), m->d_out, train ? m->d_h2f : nullptr, m->d_gcols, m->d_rowloss, m->d_dh2b);
    TA3W_CUDA(m, cudaGetLastError(), "head");
    if (!train) return 0;
    // dW2 = dH2^T H1 (M = h out, N = h in, K = rows), straight into the gradient vector
    if (gemm(m, 1, 1, m->d_dh2b, h, nullptr, m->d_h1b, h, nullptr, m->d_grad + d.w2, h, 0, h, h, R, 1)) return 1;
    // F3 = dH2 W2 (M = rows, N = h in, K = h out), then the ReLU mask of layer 1
    if (gemm(m, 0, 1, m->d_dh2b, h, nullptr, m->d_w2b, h, nullptr, m->d_f2, h, 0, R, h, h, 1)) return 1;
    mask1_kernel<<<unsigned((n_act + 255) / 256), 256, 0, m->stream>>>(m->d_f2, m->d_h1b, n_act, m->d_dh1b);
    TA3W_CUDA(m, cudaGetLastError(), "mask1");
    // dW1 = dH1^T X (M = h, N = inp, K = rows)
    if (gemm(m, 1, 1, m->d_dh1b, h, nullptr, m->d_x, d.inp, rows, m->d_grad + d.w1, d.inp, 0, h, d.inp, R, 1)) return 1;
    small_grads_kernel<<<unsigned((h + 3 + 127) / 128), 128, 0, m->stream>>>(
        R, h, m->d_dh1b, m->d_dh2b, m->d_h2f, m->d_gcols, m->d_rowloss, m->d_grad, d.w3, d.b1, d.b2, d.b3,
        m->d_loss);
    TA3W_CUDA(m, cudaGetLastError(), "small grads");
    return 0;
}

int check_status(ta3w_model* m) {
    uint32_t st = 0;
    TA3W_CUDA(m, cudaMemcpyAsync(&st, m->d_status, 4, cudaMemcpyDeviceToHost, m->stream), "status");
    TA3W_CUDA(m, cudaStreamSynchronize(m->stream), "surrogate kernels");
    if (st) return wfail(m, "surrogate: a tensor-core wait timed out");
    return 0;
}

int upload_rows(ta3w_model* m, float const* x, uint32_t n) {
    Dims const& d = m->d;
    if (n > m->cap_rows) {
        size_t c1 = 0, c2 = 0, c3 = 0;
        if (m->d_xraw) cudaFree(m->d_xraw);
        if (m->d_x) cudaFree(m->d_x);
        if (m->d_y) cudaFree(m->d_y);
        m->d_xraw = nullptr;
        m->d_x = nullptr;
        m->d_y = nullptr;
        m->cap_rows = 0;
        if (wgrow(m, m->d_xraw, c1, size_t(n) * d.in, "alloc rows") ||
            wgrow(m, m->d_x, c2, size_t(n) * d.inp, "alloc rows") || wgrow(m, m->d_y, c3, n, "alloc targets"))
            return 1;
        m->cap_rows = n;
    }
    TA3W_CUDA(m, cudaMemcpyAsync(m->d_xraw, x, size_t(n) * d.in * 4, cudaMemcpyHostToDevice, m->stream), "copy rows");
    int64_t const total = int64_t(n) * d.inp;
    pack_kernel<<<unsigned((total + 255) / 256), 256, 0, m->stream>>>(m->d_xraw, int(n), d.in, d.inp, m->d_stats,
                                                                      m->d_stats + d.inp, m->d_x);
    TA3W_CUDA(m, cudaGetLastError(), "pack");
    return 0;
}

} // namespace

extern "C" {

uint32_t ta3w_num_params(uint32_t in_dim, uint32_t hidden) {
    if (in_dim == 0 || hidden == 0 || hidden % TILE) return 0;
    return uint32_t(make_dims(int(in_dim), int(hidden)).n);
}

ta3w_model* ta3w_create(int device, uint32_t in_dim, uint32_t hidden, uint32_t seed) {
    if (in_dim == 0 || in_dim > (1u << 20) || hidden == 0 || hidden % TILE || hidden > 1024) {
        g_werr = "ta3w_create: in_dim in 1..2^20, hidden a multiple of 128 up to 1024";
        return nullptr;
    }
    auto* m = new ta3w_model;
    m->device = device;
    m->d = make_dims(int(in_dim), int(hidden));
    auto bad = [&](std::string what) {
        g_werr = "ta3w_create: " + what;
        ta3w_destroy(m);
        return static_cast<ta3w_model*>(nullptr);
    };
    cudaDeviceProp prop{};
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return bad("no such device");
    if (prop.major != 10) return bad("needs an sm_100 (B200) device");
    m->sms = prop.multiProcessorCount;
    m->max_splits = 16;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            if (cudaFuncSetAttribute(gemm_fn(a, b), cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_BYTES)) !=
                cudaSuccess)
                return bad("smem attribute");
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return bad("stream");
    Dims const& d = m->d;
    size_t const np = size_t(d.n);
    if (walloc(m, m->d_param, np, "params") || walloc(m, m->d_m, np, "adam m") || walloc(m, m->d_v, np, "adam v") ||
        walloc(m, m->d_grad, np, "grad") || walloc(m, m->d_w1b, size_t(d.h) * d.inp, "w1 bf16") ||
        walloc(m, m->d_w2b, size_t(d.h) * d.h, "w2 bf16") || walloc(m, m->d_status, 1, "status") ||
        walloc(m, m->d_loss, 2, "loss") || walloc(m, m->d_stats, 2 * size_t(d.inp), "stats"))
        return bad(m->err);
    // He-uniform init for the ReLU layers, small output layer (mt19937 + uniform_real_distribution)
    std::mt19937 rng(seed);
    auto uni = [&](float a) { return std::uniform_real_distribution<float>(-a, a)(rng); };
    std::vector<float> w(np, 0.f);
    for (int o = 0; o < d.h; ++o)
        for (int i = 0; i < d.in; ++i) w[size_t(d.w1) + size_t(o) * d.inp + i] = uni(std::sqrt(6.f / float(d.in)));
    for (int64_t k = 0; k < int64_t(d.h) * d.h; ++k) w[size_t(d.w2 + k)] = uni(std::sqrt(6.f / float(d.h)));
    for (int k = 0; k < 2 * d.h; ++k) w[size_t(d.w3) + k] = uni(std::sqrt(1.f / float(d.h)));
    if (ta3w_set_params(m, w.data())) return bad(m->err);
    std::vector<float> stats(2 * size_t(d.inp), 0.f);
    std::fill(stats.begin() + d.inp, stats.end(), 1.f);
    m->x_mean.assign(size_t(d.in), 0.f);
    m->x_inv_std.assign(size_t(d.in), 1.f);
    // on the model's stream: its kernels run on a non-blocking stream, which does not wait for the
    // legacy default stream (a pageable cudaMemcpy can even return before its DMA has landed)
    if (cudaMemcpyAsync(m->d_stats, stats.data(), stats.size() * 4, cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_status, 0, 4, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess)
        return bad("init copies");
    return m;
}

void ta3w_destroy(ta3w_model* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    for (void* p : {(void*)m->d_param, (void*)m->d_m, (void*)m->d_v, (void*)m->d_grad, (void*)m->d_w1b,
                    (void*)m->d_w2b, (void*)m->d_status, (void*)m->d_loss, (void*)m->d_stats, (void*)m->d_xraw,
                    (void*)m->d_x, (void*)m->d_y, (void*)m->d_idx, (void*)m->d_f1, (void*)m->d_h1b, (void*)m->d_f2,
                    (void*)m->d_h2f, (void*)m->d_gcols, (void*)m->d_rowloss, (void*)m->d_dh2b, (void*)m->d_dh1b,
                    (void*)m->d_out, (void*)m->d_rowidx})
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

const char* ta3w_last_error(const ta3w_model* m) { return m ? m->err.c_str() : g_werr.c_str(); }

uint32_t ta3w_model_params(const ta3w_model* m) { return m ? uint32_t(m->d.n) : 0u; }

int ta3w_set_params(ta3w_model* m, const float* params) {
    if (!m || !params) return wfail(m, "ta3w_set_params: null argument");
    Dims const& d = m->d;
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    std::vector<float> p(params, params + d.n);
    for (int o = 0; o < d.h; ++o)       // padding columns of W1 stay zero
        for (int i = d.in; i < d.inp; ++i) p[size_t(d.w1) + size_t(o) * d.inp + i] = 0.f;
    // on the model's (non-blocking) stream, ahead of the refresh kernel that reads them
    TA3W_CUDA(m, cudaMemcpyAsync(m->d_param, p.data(), size_t(d.n) * 4, cudaMemcpyHostToDevice, m->stream), "params");
    TA3W_CUDA(m, cudaMemsetAsync(m->d_m, 0, size_t(d.n) * 4, m->stream), "adam m");
    TA3W_CUDA(m, cudaMemsetAsync(m->d_v, 0, size_t(d.n) * 4, m->stream), "adam v");
    m->adam_t = 0;
    refresh_kernel<<<unsigned((d.w3 + 255) / 256), 256, 0, m->stream>>>(m->d_param, d.w2, d.w3, m->d_w1b, m->d_w2b);
    TA3W_CUDA(m, cudaGetLastError(), "refresh");
    TA3W_CUDA(m, cudaStreamSynchronize(m->stream), "refresh");
    return 0;
}

int ta3w_get_params(ta3w_model* m, float* params_out) {
    if (!m || !params_out) return wfail(m, "ta3w_get_params: null argument");
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    TA3W_CUDA(m, cudaStreamSynchronize(m->stream), "sync");
    TA3W_CUDA(m, cudaMemcpy(params_out, m->d_param, size_t(m->d.n) * 4, cudaMemcpyDeviceToHost), "params");
    return 0;
}

static int set_data_impl(ta3w_model* m, const float* x, const float* y, uint32_t n, bool standardize) {
    Dims const& d = m->d;
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    std::vector<float> stats(2 * size_t(d.inp), 0.f);
    std::fill(stats.begin() + d.inp, stats.end(), 1.f);
    m->y_mean = 0.f;
    m->y_std = 1.f;
    if (standardize) {
        for (int c = 0; c < d.in; ++c) {
            double s = 0, s2 = 0;
            for (uint32_t r = 0; r < n; ++r) s += x[size_t(r) * d.in + c];
            double const mu = s / n;
            for (uint32_t r = 0; r < n; ++r) {
                double const dv = x[size_t(r) * d.in + c] - mu;
                s2 += dv * dv;
            }
            double const sd = std::sqrt(s2 / n);
            m->x_mean[c] = float(mu);
            m->x_inv_std[c] = sd > 1e-12 ? float(1.0 / sd) : 1.f;
            stats[c] = m->x_mean[c];
            stats[d.inp + c] = m->x_inv_std[c];
        }
        double s = 0, s2 = 0;
        for (uint32_t r = 0; r < n; ++r) s += y[r];
        double const mu = s / n;
        for (uint32_t r = 0; r < n; ++r) s2 += (y[r] - mu) * (y[r] - mu);
        m->y_mean = float(mu);
        m->y_std = s2 > 0 ? float(std::sqrt(s2 / n)) : 1.f;
    } else {
        std::fill(m->x_mean.begin(), m->x_mean.end(), 0.f);
        std::fill(m->x_inv_std.begin(), m->x_inv_std.end(), 1.f);
    }
    TA3W_CUDA(m, cudaMemcpyAsync(m->d_stats, stats.data(), stats.size() * 4, cudaMemcpyHostToDevice, m->stream),
              "stats");
    if (upload_rows(m, x, n)) return 1;
    std::vector<float> ys(n);
    for (uint32_t r = 0; r < n; ++r) ys[r] = (y[r] - m->y_mean) / m->y_std;
    TA3W_CUDA(m, cudaMemcpyAsync(m->d_y, ys.data(), size_t(n) * 4, cudaMemcpyHostToDevice, m->stream), "targets");
    TA3W_CUDA(m, cudaStreamSynchronize(m->stream), "set data");
    m->rows = n;
    return 0;
}

int ta3w_set_data(ta3w_model* m, const float* x, const float* y, uint32_t n) {
    if (!m || !x || !y || n == 0) return wfail(m, "ta3w_set_data: need n > 0 rows");
    return set_data_impl(m, x, y, n, true);
}

int ta3w_set_data_standardized(ta3w_model* m, const float* x, const float* y, uint32_t n) {
    if (!m || !x || !y || n == 0) return wfail(m, "ta3w_set_data_standardized: need n > 0 rows");
    return set_data_impl(m, x, y, n, false);
}

int ta3w_gradients(ta3w_model* m, float* grad_out, float* loss_sum_out) {
    if (!m || !grad_out) return wfail(m, "ta3w_gradients: null argument");
    if (m->rows == 0) return wfail(m, "ta3w_gradients: no data");
    if (m->rows > kMaxPassRows) return wfail(m, "ta3w_gradients: at most 65,536 rows in one pass");
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    TA3W_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    TA3W_CUDA(m, cudaMemsetAsync(m->d_grad, 0, size_t(m->d.n) * 4, m->stream), "grad");
    if (pass(m, nullptr, int(m->rows), true)) return 1;
    if (check_status(m)) return 1;
    TA3W_CUDA(m, cudaMemcpy(grad_out, m->d_grad, size_t(m->d.n) * 4, cudaMemcpyDeviceToHost), "grad");
    if (loss_sum_out) TA3W_CUDA(m, cudaMemcpy(loss_sum_out, m->d_loss, 4, cudaMemcpyDeviceToHost), "loss");
    return 0;
}

int ta3w_train(ta3w_model* m, uint32_t epochs, uint32_t batch, float lr, float weight_decay, uint32_t seed,
               float* final_loss) {
    if (!m || batch == 0 || batch > kMaxPassRows) return wfail(m, "ta3w_train: batch must be 1 .. 65,536");
    if (m->rows == 0) return wfail(m, "ta3w_train: no data");
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    Dims const& d = m->d;
    uint32_t const n = m->rows;
    uint32_t const steps = (n + batch - 1) / batch;
    size_t const total = size_t(epochs) * steps * batch;
    std::vector<int32_t> idx(std::max<size_t>(total, 1), -1);
    std::mt19937 rng(seed);
    std::vector<int32_t> perm(n);
    for (uint32_t e = 0; e < epochs; ++e) {
        std::iota(perm.begin(), perm.end(), 0);
        std::shuffle(perm.begin(), perm.end(), rng);
        for (uint32_t s = 0; s < steps; ++s)
            for (uint32_t b = 0; b < batch; ++b) {
                uint32_t const k = s * batch + b;
                idx[(size_t(e) * steps + s) * batch + b] = k < n ? perm[k] : -1;
            }
    }
    if (wgrow(m, m->d_idx, m->cap_idx, idx.size(), "alloc indices")) return 1;
    TA3W_CUDA(m, cudaMemcpyAsync(m->d_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, m->stream), "indices");
    TA3W_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float last_loss = 0.f;
    uint32_t last_rows = 0;
    for (uint32_t e = 0; e < epochs; ++e)
        for (uint32_t s = 0; s < steps; ++s) {
            uint32_t const rows_here = std::min(batch, n - s * batch);
            if (pass(m, m->d_idx + (size_t(e) * steps + s) * batch, int(rows_here), true)) return 1;
            ++m->adam_t;
            float const c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
            adam_kernel<<<unsigned((d.n + 255) / 256), 256, 0, m->stream>>>(
                m->d_param, m->d_m, m->d_v, m->d_grad, d.n, d.w2, d.w3, d.in, d.inp, lr, b1, b2, eps, c1, c2,
                weight_decay, m->d_w1b, m->d_w2b);
            TA3W_CUDA(m, cudaGetLastError(), "adam");
            last_rows = rows_here;
        }
    if (check_status(m)) return 1;
    if (final_loss) {
        TA3W_CUDA(m, cudaMemcpy(&last_loss, m->d_loss, 4, cudaMemcpyDeviceToHost), "loss");
        *final_loss = last_rows ? last_loss / float(last_rows) : 0.f;
    }
    return 0;
}

int ta3w_predict(ta3w_model* m, const float* x, uint32_t n, float* mean_out, float* logvar_out) {
    if (!m || !x || !mean_out) return wfail(m, "ta3w_predict: null argument");
    if (n == 0) return 0;
    TA3W_CUDA(m, cudaSetDevice(m->device), "set device");
    if (upload_rows(m, x, n)) return 1;
    TA3W_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    uint32_t const chunk = 4096;
    std::vector<float> out(size_t(n) * 2);
    for (uint32_t r0 = 0; r0 < n; r0 += chunk) {
        uint32_t const k = std::min(chunk, n - r0);
        std::vector<int32_t> map(k);
        std::iota(map.begin(), map.end(), int32_t(r0));
        size_t cap = m->cap_idx;
        if (wgrow(m, m->d_idx, cap, std::max<size_t>(m->cap_idx, k), "alloc indices")) return 1;
        m->cap_idx = cap;
        TA3W_CUDA(m, cudaMemcpyAsync(m->d_idx, map.data(), size_t(k) * 4, cudaMemcpyHostToDevice, m->stream), "rows");
        if (pass(m, m->d_idx, int(k), false)) return 1;
        TA3W_CUDA(m, cudaMemcpyAsync(out.data() + size_t(r0) * 2, m->d_out, size_t(k) * 8, cudaMemcpyDeviceToHost,
                                     m->stream), "outputs");
        TA3W_CUDA(m, cudaStreamSynchronize(m->stream), "predict");
    }
    if (check_status(m)) return 1;
    for (uint32_t r = 0; r < n; ++r) {
        mean_out[r] = out[2 * r] * m->y_std + m->y_mean;
        if (logvar_out) logvar_out[r] = out[2 * r + 1] + 2.f * std::log(m->y_std);
    }
    m->rows = 0;   // the training rows were overwritten: a later train call needs set_data again
    return 0;
}

// Test hook: C = A B^T-style product of the GEMM kernel on host BF16 data (bit
// patterns as uint16), both operands given in their global layouts; c [m][n].
int ta3w_gemm_test(int device, int a_mn, int b_mn, int m, int n, int k, int splits, const uint16_t* a,
                   const uint16_t* b, float* c) {
    if (m <= 0 || n <= 0 || k <= 0 || m % TILE || n % TILE || k % KS || splits < 1) {
        g_werr = "ta3w_gemm_test: m, n multiples of 128, k of 64";
        return 1;
    }
    ta3w_model tmp;
    tmp.device = device;
    ta3w_model* mm = &tmp;
    TA3W_CUDA(mm, cudaSetDevice(device), "set device");
    cudaDeviceProp prop{};
    TA3W_CUDA(mm, cudaGetDeviceProperties(&prop, device), "properties");
    if (prop.major != 10) return wfail(mm, "needs an sm_100 device");
    tmp.sms = prop.multiProcessorCount;
    TA3W_CUDA(mm, cudaFuncSetAttribute(gemm_fn(a_mn, b_mn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(SMEM_BYTES)), "smem attribute");
    __nv_bfloat16 *da = nullptr, *db = nullptr;
    float* dc = nullptr;
    uint32_t* ds = nullptr;
    int const kst = k / KS;
    int const per = (kst + splits - 1) / splits;
    int const used = (kst + per - 1) / per;
    int rc = 0;
    if (cudaMalloc(&da, size_t(m) * k * 2) != cudaSuccess || cudaMalloc(&db, size_t(n) * k * 2) != cudaSuccess ||
        cudaMalloc(&dc, size_t(used) * m * n * 4) != cudaSuccess || cudaMalloc(&ds, 4) != cudaSuccess) {
        rc = wfail(mm, "alloc");
    } else {
        cudaMemcpy(da, a, size_t(m) * k * 2, cudaMemcpyHostToDevice);
        cudaMemcpy(db, b, size_t(n) * k * 2, cudaMemcpyHostToDevice);
        cudaMemset(ds, 0, 4);
        GemmArgs g{da, a_mn ? m : k, nullptr, db, b_mn ? n : k, nullptr, dc, n, int64_t(m) * n, m, n, k, per * KS, ds};
        gemm_fn(a_mn, b_mn)<<<dim3(m / TILE, n / TILE, used), THREADS, SMEM_BYTES>>>(g);
        cudaError_t e = cudaDeviceSynchronize();
        uint32_t st = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&st, ds, 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = wfail(mm, std::string("gemm: ") + cudaGetErrorString(e));
        else if (st) rc = wfail(mm, "gemm: a tensor-core wait timed out");
        else {
            std::vector<float> part(size_t(used) * m * n);
            cudaMemcpy(part.data(), dc, part.size() * 4, cudaMemcpyDeviceToHost);
            for (size_t i = 0; i < size_t(m) * n; ++i) {
                float s = 0.f;
                for (int q = 0; q < used; ++q) s += part[size_t(q) * m * n + i];
                c[i] = s;
            }
        }
    }
    for (void* p : {(void*)da, (void*)db, (void*)dc, (void*)ds})
        if (p) cudaFree(p);
    if (rc) g_werr = tmp.err;
    return rc;
}

} // extern "C"
