// Surrogate fitness model for CMA-ES pre-screening: an MLP 97 -> 128 -> 128 -> 2
// (predicted mean score, log-variance) trained by Gaussian negative log-likelihood
// with Adam. No counterpart in the reference; the trainer calls it through
// include/ta3b_surrogate.h.
//
// Tensor-core path (sm_100a): every 128x128 GEMM of the forward and backward
// pass is a tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32
// accumulators in tensor memory) issued by one thread; the 2-wide output layer,
// the loss and the elementwise parts run on the CUDA cores from TMEM values.
// One CTA (4 warps, 128 threads, ~200 KB shared memory, all 512 TMEM columns)
// per SM; thread t owns batch row t of a 128-row tile for the elementwise work
// and TMEM lane t (= output row t of every MMA).
//
// Shared-memory operand layout (no swizzle): a 128 x 128 BF16 tile stores
// element (r, c) at byte (r/8)*2048 + (c/8)*128 + (r%8)*16 + (c%8)*2, i.e. 8x8
// "core matrices" of 128 contiguous bytes. The same bytes read as
//   K-major with rows as M/N:  LBO = 128 (next 8 columns), SBO = 2048 (next 8 rows)
//   MN-major with rows as K:   LBO = 2048 (next 8 rows = K), SBO = 128 (next 8 columns = M/N)
// so an activation tile written once by its row owners serves both as the
// A operand of a row-major GEMM (M = batch) and as an operand of the weight
// gradient GEMMs (K = batch) without a transpose.
//
// Descriptor encodings follow the PTX ISA tcgen05 shared-memory and instruction
// descriptors (field layout as in CUTLASS cute/arch/mma_sm100_desc.hpp).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/ta3b_surrogate.h"

namespace ta3s {

constexpr int IN = 97;          // v11 parameter count
constexpr int IN_K = 112;       // first-layer K, padded to a multiple of 16
constexpr int HID = 128;
constexpr int ROWS = 128;       // batch rows per tile = MMA M
constexpr int THREADS = 128;

// flat FP32 parameter vector (also the gradient layout)
constexpr int OFF_W1 = 0;                       // [128][112] (o, i); i >= 97 stays zero
constexpr int OFF_W2 = OFF_W1 + HID * IN_K;     // [128][128] (o, i)
constexpr int OFF_W3 = OFF_W2 + HID * HID;      // [2][128]
constexpr int OFF_B1 = OFF_W3 + 2 * HID;
constexpr int OFF_B2 = OFF_B1 + HID;
constexpr int OFF_B3 = OFF_B2 + HID;
constexpr int NPARAM = OFF_B3 + 2;              // 31234
constexpr int PARTIAL = NPARAM + 2;             // + loss sum + valid rows

// shared memory map (bytes from a 1024-aligned base)
constexpr uint32_t TILE_BYTES = 128 * 128 * 2;
constexpr uint32_t S_X = 0, S_W1 = S_X + TILE_BYTES, S_W2 = S_W1 + TILE_BYTES, S_H1 = S_W2 + TILE_BYTES,
                   S_H2 = S_H1 + TILE_BYTES, S_D1 = S_H2 + TILE_BYTES, S_G = S_D1 + TILE_BYTES;   // S_G: [128][16]
constexpr uint32_t S_F32 = S_G + 128 * 16 * 2;  // W3 [2][128], b1, b2 [128], b3 [2]
constexpr uint32_t S_BAR = S_F32 + (4 * HID + 4) * 4;
constexpr uint32_t S_TMEM = S_BAR + 8;
constexpr uint32_t SMEM_BYTES = S_TMEM + 8 + 1024;   // + alignment slack

// TMEM columns
constexpr uint32_t T_F1 = 0, T_F2 = 128, T_DW2 = 256, T_DW1 = 384, T_SMALL = 496;

constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL;   // ~2 s at 1.9 GHz

__host__ __device__ constexpr uint32_t tile_off(int r, int c) {
    return uint32_t((r >> 3) * 2048 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}
__host__ __device__ constexpr uint32_t gtile_off(int r, int c) {   // [128][16] tile
    return uint32_t((r >> 3) * 256 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// tcgen05 shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

// instruction descriptor: D F32, A/B BF16, majors (0 = K, 1 = MN), N, M = 128
__host__ __device__ constexpr uint32_t instr_desc(int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           (uint32_t(n >> 3) << 17) | (uint32_t(ROWS >> 4) << 24);
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

// 16 consecutive FP32 columns of this thread's TMEM lane
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

// bounded wait for the barrier phase with the given parity; false on timeout
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

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 const h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t const*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// 8 FP32 values -> one 16-byte BF16 chunk of a tile
__device__ __forceinline__ void st_chunk(uint8_t* smem, uint32_t off, float const* v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(smem + off) = q;
}

struct Params {
    __nv_bfloat16 const* x;     // [rows][128] standardised inputs (columns >= 97 zero)
    float const* y;             // [rows] standardised targets (training)
    int32_t const* idx;         // batch row indices, or null for rows 0..batch-1
    int batch;
    __nv_bfloat16 const* w1;    // [128][128] (o, i), i >= 97 zero
    __nv_bfloat16 const* w2;    // [128][128] (o, i)
    float const* p32;           // FP32 parameters (W3 and biases read from here)
    float* out;                 // prediction: [batch][2]
    float* partial;             // training: [gridDim.x][PARTIAL]
    uint32_t* status;           // nonzero: a tensor-core wait timed out
    float inv_batch;
    int train;
};

__global__ void __launch_bounds__(THREADS, 1) mlp_kernel(Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint32_t const sbase = uint32_t(__cvta_generic_to_shared(sm));
    int const tid = threadIdx.x, warp = tid >> 5;
    float* w3s = reinterpret_cast<float*>(sm + S_F32);
    float* b1s = w3s + 2 * HID;
    float* b2s = b1s + HID;
    float* b3s = b2s + HID;
    uint32_t const bar = sbase + S_BAR;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + S_TMEM);
    volatile uint32_t* abort_s = reinterpret_cast<volatile uint32_t*>(sm + S_TMEM + 4);   // block-uniform stop

    // weights into shared memory: thread o owns rows o of W1 and W2
    for (int c = 0; c < 16; ++c) {
        *reinterpret_cast<uint4*>(sm + S_W1 + tile_off(tid, c * 8)) =
            __ldg(reinterpret_cast<uint4 const*>(p.w1 + tid * 128 + c * 8));
        *reinterpret_cast<uint4*>(sm + S_W2 + tile_off(tid, c * 8)) =
            __ldg(reinterpret_cast<uint4 const*>(p.w2 + tid * 128 + c * 8));
    }
    w3s[tid] = p.p32[OFF_W3 + tid];
    w3s[HID + tid] = p.p32[OFF_W3 + HID + tid];
    b1s[tid] = p.p32[OFF_B1 + tid];
    b2s[tid] = p.p32[OFF_B2 + tid];
    if (tid < 2) b3s[tid] = p.p32[OFF_B3 + tid];
    if (tid == 0) {
        mbar_init(bar);
        *abort_s = 0u;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + S_TMEM),
                     "r"(512u) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    uint32_t const tmem = *tmem_slot;
    uint32_t const lane_base = tmem + (uint32_t(warp * 32) << 16);   // this warp's TMEM lanes
    uint32_t phase = 0;
    bool ok = true;

    // every thread waits for the last commit; a timeout is recorded and makes the
    // whole block stop at the next tile boundary (all threads read the flag after a barrier)
    auto sync_mma = [&]() {
        if (ok && !mbar_wait(bar, phase)) {
            ok = false;
            *abort_s = 1u;
            atomicOr(p.status, 1u);
        }
        phase ^= 1u;
        fence_after();
    };
    auto publish = [&]() {           // smem writes + TMEM reads done -> MMA may run
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
    };

    uint32_t const x_s = sbase + S_X, w1_s = sbase + S_W1, w2_s = sbase + S_W2, h1_s = sbase + S_H1,
                   h2_s = sbase + S_H2, d1_s = sbase + S_D1, g_s = sbase + S_G;
    uint32_t const id128_kk = instr_desc(128, 0, 0), id128_mm = instr_desc(128, 1, 1),
                   id128_km = instr_desc(128, 0, 1), id112_mm = instr_desc(IN_K, 1, 1),
                   id16_mm = instr_desc(16, 1, 1);

    float acc_w3a = 0.f, acc_w3b = 0.f, acc_b1 = 0.f, acc_b2 = 0.f;   // lane = feature
    float acc_b3a = 0.f, acc_b3b = 0.f, acc_loss = 0.f, acc_rows = 0.f;   // row owner
    int const ntiles = (p.batch + ROWS - 1) / ROWS;
    bool first = true;

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        int const r = tile * ROWS + tid;
        bool const valid = r < p.batch;
        int const row = valid ? (p.idx ? p.idx[r] : r) : 0;
        // ---- X tile
        for (int c = 0; c < 16; ++c) {
            uint4 q = make_uint4(0, 0, 0, 0);
            if (valid) q = __ldg(reinterpret_cast<uint4 const*>(p.x + size_t(row) * 128 + c * 8));
            *reinterpret_cast<uint4*>(sm + S_X + tile_off(tid, c * 8)) = q;
        }
        float const yv = (p.train && valid) ? p.y[row] : 0.f;
        publish();
        // ---- layer 1: H1 = X W1^T (M = rows, N = 128, K = 112)
        if (tid == 0) {
            for (int kk = 0; kk < IN_K / 16; ++kk)
                mma_bf16(tmem + T_F1, smem_desc(x_s + kk * 256, 128, 2048), smem_desc(w1_s + kk * 256, 128, 2048),
                         id128_kk, kk > 0);
            mma_commit(bar);
        }
        sync_mma();
        for (int cc = 0; cc < 8; ++cc) {
            float v[16];
            tmem_ld16(lane_base + T_F1 + cc * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + b1s[cc * 16 + j], 0.f);
            st_chunk(sm + S_H1, tile_off(tid, cc * 16), v);
            st_chunk(sm + S_H1, tile_off(tid, cc * 16 + 8), v + 8);
        }
        publish();
        // ---- layer 2: H2 = relu(H1) W2^T
        if (tid == 0) {
            for (int kk = 0; kk < HID / 16; ++kk)
                mma_bf16(tmem + T_F2, smem_desc(h1_s + kk * 256, 128, 2048), smem_desc(w2_s + kk * 256, 128, 2048),
                         id128_kk, kk > 0);
            mma_commit(bar);
        }
        sync_mma();
        // ---- output layer on the CUDA cores (FP32): mean, log-variance
        float o0 = b3s[0], o1 = b3s[1];
        for (int cc = 0; cc < 8; ++cc) {
            float v[16];
            tmem_ld16(lane_base + T_F2 + cc * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float const h = fmaxf(v[j] + b2s[cc * 16 + j], 0.f);
                v[j] = h;
                o0 = fmaf(h, w3s[cc * 16 + j], o0);
                o1 = fmaf(h, w3s[HID + cc * 16 + j], o1);
            }
            if (p.train) {
                st_chunk(sm + S_H2, tile_off(tid, cc * 16), v);
                st_chunk(sm + S_H2, tile_off(tid, cc * 16 + 8), v + 8);
            }
        }
        if (!p.train) {
            if (valid) {
                p.out[size_t(r) * 2] = o0;
                p.out[size_t(r) * 2 + 1] = o1;
            }
            fence_before();
            __syncthreads();
            fence_after();
            ok = *abort_s == 0u;
            continue;
        }
        // ---- Gaussian NLL 0.5 * (s + (y - mu)^2 e^-s), mean over the batch
        float dmu = 0.f, ds = 0.f;
        if (valid) {
            float const s = fminf(fmaxf(o1, -12.f), 12.f);
            float const e = expf(-s);
            float const d = yv - o0;
            acc_loss += 0.5f * (s + d * d * e);
            acc_rows += 1.f;
            dmu = -d * e * p.inv_batch;
            ds = (o1 > -12.f && o1 < 12.f) ? 0.5f * (1.f - d * d * e) * p.inv_batch : 0.f;
        }
        acc_b3a += dmu;
        acc_b3b += ds;
        {
            float g[16] = {valid ? 1.f : 0.f, dmu, ds, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            st_chunk(sm + S_G, gtile_off(tid, 0), g);
            st_chunk(sm + S_G, gtile_off(tid, 8), g + 8);
        }
        publish();
        // ---- dW3^T[i][c] = sum_b H2[b][i] G[b][c]   (M = feature, N = 16, K = rows)
        if (tid == 0) {
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma_bf16(tmem + T_SMALL, smem_desc(h2_s + kk * 4096, 2048, 128), smem_desc(g_s + kk * 512, 256, 128),
                         id16_mm, kk > 0);
            mma_commit(bar);
        }
        sync_mma();
        {
            float v[16];
            tmem_ld16(lane_base + T_SMALL, v);
            acc_w3a += v[1];
            acc_w3b += v[2];
        }
        // ---- dH2 = (dmu W3[0] + ds W3[1]) * relu'(H2) (overwrites the H2 tile: its MMA has completed)
        for (int cc = 0; cc < 8; ++cc) {
            float v[16];
            tmem_ld16(lane_base + T_F2 + cc * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                int const o = cc * 16 + j;
                v[j] = (v[j] + b2s[o] > 0.f) ? fmaf(dmu, w3s[o], ds * w3s[HID + o]) : 0.f;
            }
            st_chunk(sm + S_H2, tile_off(tid, cc * 16), v);
            st_chunk(sm + S_H2, tile_off(tid, cc * 16 + 8), v + 8);
        }
        publish();
        // ---- dW2 += dH2^T H1, dH1 = dH2 W2, db2 = column sums of dH2
        if (tid == 0) {
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma_bf16(tmem + T_DW2, smem_desc(h2_s + kk * 4096, 2048, 128), smem_desc(h1_s + kk * 4096, 2048, 128),
                         id128_mm, (!first || kk > 0) ? 1u : 0u);
            for (int kk = 0; kk < HID / 16; ++kk)
                mma_bf16(tmem + T_F1, smem_desc(h2_s + kk * 256, 128, 2048), smem_desc(w2_s + kk * 4096, 2048, 128),
                         id128_km, kk > 0);
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma_bf16(tmem + T_SMALL, smem_desc(h2_s + kk * 4096, 2048, 128), smem_desc(g_s + kk * 512, 256, 128),
                         id16_mm, kk > 0);
            mma_commit(bar);
        }
        sync_mma();
        {
            float v[16];
            tmem_ld16(lane_base + T_SMALL, v);
            acc_b2 += v[0];
        }
        // ---- dH1 = (dH2 W2) * relu'(H1), the mask read back from this thread's H1 row
        for (int cc = 0; cc < 8; ++cc) {
            float v[16];
            tmem_ld16(lane_base + T_F1 + cc * 16, v);
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                uint4 const h = *reinterpret_cast<uint4 const*>(sm + S_H1 + tile_off(tid, cc * 16 + half * 8));
                uint32_t const hw[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float* vv = v + half * 8 + q * 2;
                    if (!(bf16_lo(hw[q]) > 0.f)) vv[0] = 0.f;
                    if (!(bf16_hi(hw[q]) > 0.f)) vv[1] = 0.f;
                }
            }
            st_chunk(sm + S_D1, tile_off(tid, cc * 16), v);
            st_chunk(sm + S_D1, tile_off(tid, cc * 16 + 8), v + 8);
        }
        publish();
        // ---- dW1 += dH1^T X (N = 112), db1 = column sums of dH1
        if (tid == 0) {
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma_bf16(tmem + T_DW1, smem_desc(d1_s + kk * 4096, 2048, 128), smem_desc(x_s + kk * 4096, 2048, 128),
                         id112_mm, (!first || kk > 0) ? 1u : 0u);
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma_bf16(tmem + T_SMALL, smem_desc(d1_s + kk * 4096, 2048, 128), smem_desc(g_s + kk * 512, 256, 128),
                         id16_mm, kk > 0);
            mma_commit(bar);
        }
        sync_mma();
        {
            float v[16];
            tmem_ld16(lane_base + T_SMALL, v);
            acc_b1 += v[0];
        }
        first = false;
        fence_before();
        __syncthreads();
        fence_after();
        ok = *abort_s == 0u;
    }

    if (p.train) {
        float* part = p.partial + size_t(blockIdx.x) * PARTIAL;
        int const o = tid;   // TMEM lane = feature row of the weight gradients
        if (ok && !first) {
            for (int cc = 0; cc < 8; ++cc) {
                float v[16];
                tmem_ld16(lane_base + T_DW2 + cc * 16, v);
                for (int j = 0; j < 16; ++j) part[OFF_W2 + o * HID + cc * 16 + j] = v[j];
            }
            for (int cc = 0; cc < IN_K / 16; ++cc) {
                float v[16];
                tmem_ld16(lane_base + T_DW1 + cc * 16, v);
                for (int j = 0; j < 16; ++j) part[OFF_W1 + o * IN_K + cc * 16 + j] = (cc * 16 + j < IN) ? v[j] : 0.f;
            }
        } else {
            for (int i = 0; i < HID; ++i) part[OFF_W2 + o * HID + i] = 0.f;
            for (int i = 0; i < IN_K; ++i) part[OFF_W1 + o * IN_K + i] = 0.f;
        }
        part[OFF_W3 + o] = acc_w3a;
        part[OFF_W3 + HID + o] = acc_w3b;
        part[OFF_B1 + o] = acc_b1;
        part[OFF_B2 + o] = acc_b2;
        // row-owned sums: block reduction through shared memory (the S_G tile is free now)
        float* red = reinterpret_cast<float*>(sm + S_G);
        __syncthreads();
        red[tid] = acc_b3a;
        red[THREADS + tid] = acc_b3b;
        red[2 * THREADS + tid] = acc_loss;
        red[3 * THREADS + tid] = acc_rows;
        __syncthreads();
        if (tid < 4) {
            float s = 0.f;
            for (int k = 0; k < THREADS; ++k) s += red[tid * THREADS + k];
            int const dst[4] = {OFF_B3, OFF_B3 + 1, NPARAM, NPARAM + 1};
            part[dst[tid]] = s;
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
}

// Adam over the flat parameter vector; gradients summed over the CTA partials
// in a fixed order (deterministic). Refreshes the BF16 weight copies.
__global__ void adam_kernel(float* __restrict__ param, float* __restrict__ m, float* __restrict__ v,
                            float const* __restrict__ partial, int nparts, float lr, float b1, float b2, float eps,
                            float c1, float c2, float wd, __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b,
                            float* __restrict__ loss_out) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < PARTIAL && i >= NPARAM && loss_out) {
        float s = 0.f;
        for (int k = 0; k < nparts; ++k) s += partial[size_t(k) * PARTIAL + i];
        loss_out[i - NPARAM] = s;
    }
    if (i >= NPARAM) return;
    float g = 0.f;
    for (int k = 0; k < nparts; ++k) g += partial[size_t(k) * PARTIAL + i];
    bool const pad = i < OFF_W2 && (i % IN_K) >= IN;
    if (pad) return;
    float const mi = b1 * m[i] + (1.f - b1) * g;
    float const vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float const w = param[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps) - lr * wd * param[i];   // AdamW
    param[i] = w;
    if (i < OFF_W2) {
        int const o = i / IN_K, c = i % IN_K;
        w1b[o * 128 + c] = __float2bfloat16_rn(w);
    } else if (i < OFF_W3) {
        int const k = i - OFF_W2;
        w2b[k] = __float2bfloat16_rn(w);
    }
}

// BF16 weight copies from the FP32 parameters
__global__ void refresh_kernel(float const* __restrict__ param, __nv_bfloat16* __restrict__ w1b,
                               __nv_bfloat16* __restrict__ w2b) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 128 * 128) {
        int const o = i / 128, c = i % 128;
        w1b[i] = __float2bfloat16_rn(c < IN ? param[OFF_W1 + o * IN_K + c] : 0.f);
        w2b[i] = __float2bfloat16_rn(param[OFF_W2 + i]);
    }
}

// standardised FP32 rows -> BF16 [rows][128]
__global__ void pack_kernel(float const* __restrict__ x, int rows, float const* __restrict__ mean,
                            float const* __restrict__ inv_std, __nv_bfloat16* __restrict__ xb) {
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * 128) return;
    int const r = i / 128, c = i % 128;
    float const v = c < IN ? (x[size_t(r) * IN + c] - mean[c]) * inv_std[c] : 0.f;
    xb[i] = __float2bfloat16_rn(v);
}

} // namespace ta3s

using namespace ta3s;

struct ta3s_model {
    int device = 0;
    int sms = 0;
    std::string err;
    std::mt19937 rng;
    float* d_param = nullptr;     // FP32 master parameters
    float* d_m = nullptr;
    float* d_v = nullptr;
    __nv_bfloat16* d_w1b = nullptr;
    __nv_bfloat16* d_w2b = nullptr;
    float* d_partial = nullptr;   // [sms][PARTIAL]
    uint32_t* d_status = nullptr;
    float* d_loss = nullptr;      // [2]
    // data
    size_t cap_rows = 0;
    float* d_xraw = nullptr;
    __nv_bfloat16* d_x = nullptr;
    float* d_y = nullptr;
    int32_t* d_idx = nullptr;
    size_t cap_idx = 0;
    float* d_out = nullptr;
    float* d_stats = nullptr;     // mean[128], inv_std[128]
    std::vector<float> x_mean, x_inv_std;
    float y_mean = 0.f, y_std = 1.f;
    uint32_t rows = 0;
    uint64_t adam_t = 0;
    cudaStream_t stream = nullptr;
};

namespace {
thread_local std::string g_err;

#define TA3S_CUDA(m, call, what)                                                           \
    do {                                                                                   \
        cudaError_t const e_ = (call);                                                     \
        if (e_ != cudaSuccess) return fail(m, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int fail(ta3s_model* m, std::string msg) {
    if (m) m->err = msg;
    g_err = msg;
    return 1;
}

template<class T>
int grow(ta3s_model* m, T*& ptr, size_t& cap, size_t n, char const* what) {
    if (n <= cap && ptr) return 0;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    TA3S_CUDA(m, cudaMalloc(&ptr, n * sizeof(T)), what);
    cap = n;
    return 0;
}

int check_status(ta3s_model* m) {
    uint32_t st = 0;
    TA3S_CUDA(m, cudaMemcpyAsync(&st, m->d_status, 4, cudaMemcpyDeviceToHost, m->stream), "status");
    TA3S_CUDA(m, cudaStreamSynchronize(m->stream), "surrogate kernels");
    if (st) return fail(m, "surrogate: a tensor-core wait timed out");
    return 0;
}

int upload_rows(ta3s_model* m, float const* x, uint32_t n) {
    size_t cap = m->cap_rows;
    if (n > cap) {
        size_t c1 = cap, c2 = cap, c3 = cap;
        if (grow(m, m->d_xraw, c1, size_t(n) * IN, "alloc rows") || grow(m, m->d_x, c2, size_t(n) * 128, "alloc rows") ||
            grow(m, m->d_y, c3, n, "alloc targets"))
            return 1;
        size_t c4 = cap;
        if (grow(m, m->d_out, c4, size_t(n) * 2, "alloc outputs")) return 1;
        m->cap_rows = n;
    }
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_xraw, x, size_t(n) * IN * 4, cudaMemcpyHostToDevice, m->stream), "copy rows");
    pack_kernel<<<(n * 128 + 255) / 256, 256, 0, m->stream>>>(m->d_xraw, int(n), m->d_stats, m->d_stats + 128, m->d_x);
    TA3S_CUDA(m, cudaGetLastError(), "pack");
    return 0;
}

int launch_mlp(ta3s_model* m, int batch, int32_t const* d_idx, int train) {
    int const ntiles = (batch + ROWS - 1) / ROWS;
    int const grid = std::min(ntiles, m->sms);
    Params prm{};
    prm.x = m->d_x;
    prm.y = m->d_y;
    prm.idx = d_idx;
    prm.batch = batch;
    prm.w1 = m->d_w1b;
    prm.w2 = m->d_w2b;
    prm.p32 = m->d_param;
    prm.out = m->d_out;
    prm.partial = m->d_partial;
    prm.status = m->d_status;
    prm.inv_batch = 1.0f / float(batch);
    prm.train = train;
    mlp_kernel<<<grid, THREADS, SMEM_BYTES, m->stream>>>(prm);
    TA3S_CUDA(m, cudaGetLastError(), "surrogate mlp launch");
    return 0;
}

} // namespace

extern "C" {

uint32_t ta3s_num_params(void) { return NPARAM; }

ta3s_model* ta3s_create(int device, uint32_t seed) {
    auto* m = new ta3s_model;
    m->device = device;
    m->rng.seed(seed);
    auto bad = [&](char const* what, cudaError_t e) {
        g_err = std::string("ta3s_create: ") + what + ": " + cudaGetErrorString(e);
        delete m;
        return static_cast<ta3s_model*>(nullptr);
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bad("set device", e);
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return bad("device properties", e);
    if (prop.major != 10) {
        g_err = "ta3s_create: needs an sm_100 (B200) device";
        delete m;
        return nullptr;
    }
    m->sms = prop.multiProcessorCount;
    if ((e = cudaFuncSetAttribute(mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_BYTES))) !=
        cudaSuccess)
        return bad("smem attribute", e);
    if ((e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking)) != cudaSuccess) return bad("stream", e);
    size_t const part = size_t(m->sms) * PARTIAL;
    if ((e = cudaMalloc(&m->d_param, NPARAM * 4)) != cudaSuccess || (e = cudaMalloc(&m->d_m, NPARAM * 4)) != cudaSuccess ||
        (e = cudaMalloc(&m->d_v, NPARAM * 4)) != cudaSuccess ||
        (e = cudaMalloc(&m->d_w1b, 128 * 128 * 2)) != cudaSuccess ||
        (e = cudaMalloc(&m->d_w2b, 128 * 128 * 2)) != cudaSuccess ||
        (e = cudaMalloc(&m->d_partial, part * 4)) != cudaSuccess || (e = cudaMalloc(&m->d_status, 4)) != cudaSuccess ||
        (e = cudaMalloc(&m->d_loss, 8)) != cudaSuccess || (e = cudaMalloc(&m->d_stats, 256 * 4)) != cudaSuccess)
        return bad("alloc", e);
    // He-uniform init for the ReLU layers, small output layer; FP32 master copy
    std::vector<float> w(NPARAM, 0.f);
    auto uni = [&](float a) { return std::uniform_real_distribution<float>(-a, a)(m->rng); };
    for (int o = 0; o < HID; ++o)
        for (int i = 0; i < IN; ++i) w[OFF_W1 + o * IN_K + i] = uni(std::sqrt(6.f / IN));
    for (int k = 0; k < HID * HID; ++k) w[OFF_W2 + k] = uni(std::sqrt(6.f / HID));
    for (int k = 0; k < 2 * HID; ++k) w[OFF_W3 + k] = uni(std::sqrt(1.f / HID));
    if (ta3s_set_params(m, w.data())) {
        delete m;
        return nullptr;
    }
    std::vector<float> stats(256, 0.f);
    for (int c = 0; c < 128; ++c) stats[128 + c] = 1.f;
    m->x_mean.assign(IN, 0.f);
    m->x_inv_std.assign(IN, 1.f);
    // every copy and fill goes on the model's stream: its kernels run on a non-blocking stream, which
    // does not wait for work on the legacy default stream (a pageable cudaMemcpy can even return
    // before its DMA has landed)
    if (cudaMemcpyAsync(m->d_stats, stats.data(), 256 * 4, cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_status, 0, 4, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess) {
        g_err = "ta3s_create: initial copies failed";
        ta3s_destroy(m);
        return nullptr;
    }
    return m;
}

void ta3s_destroy(ta3s_model* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    for (void* p : {(void*)m->d_param, (void*)m->d_m, (void*)m->d_v, (void*)m->d_w1b, (void*)m->d_w2b,
                    (void*)m->d_partial, (void*)m->d_status, (void*)m->d_loss, (void*)m->d_xraw, (void*)m->d_x,
                    (void*)m->d_y, (void*)m->d_idx, (void*)m->d_out, (void*)m->d_stats})
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

const char* ta3s_last_error(const ta3s_model* m) { return m ? m->err.c_str() : g_err.c_str(); }

int ta3s_set_params(ta3s_model* m, const float* params) {
    if (!m || !params) return fail(m, "ta3s_set_params: null argument");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    // on the model's (non-blocking) stream, ahead of the refresh kernel that reads them
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_param, params, NPARAM * 4, cudaMemcpyHostToDevice, m->stream), "params");
    TA3S_CUDA(m, cudaMemsetAsync(m->d_m, 0, NPARAM * 4, m->stream), "adam m");
    TA3S_CUDA(m, cudaMemsetAsync(m->d_v, 0, NPARAM * 4, m->stream), "adam v");
    m->adam_t = 0;
    refresh_kernel<<<(128 * 128 + 255) / 256, 256, 0, m->stream>>>(m->d_param, m->d_w1b, m->d_w2b);
    TA3S_CUDA(m, cudaGetLastError(), "refresh");
    TA3S_CUDA(m, cudaStreamSynchronize(m->stream), "refresh");
    return 0;
}

int ta3s_get_params(ta3s_model* m, float* params_out) {
    if (!m || !params_out) return fail(m, "ta3s_get_params: null argument");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    TA3S_CUDA(m, cudaStreamSynchronize(m->stream), "sync");
    TA3S_CUDA(m, cudaMemcpy(params_out, m->d_param, NPARAM * 4, cudaMemcpyDeviceToHost), "params");
    return 0;
}

int ta3s_set_data(ta3s_model* m, const float* x, const float* y, uint32_t n) {
    if (!m || !x || !y || n == 0) return fail(m, "ta3s_set_data: need n > 0 rows");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    // per-column standardisation of inputs and of the target (host, FP64 sums)
    std::vector<float> stats(256, 0.f);
    for (int c = 0; c < IN; ++c) {
        double s = 0, s2 = 0;
        for (uint32_t r = 0; r < n; ++r) s += x[size_t(r) * IN + c];
        double const mu = s / n;
        for (uint32_t r = 0; r < n; ++r) {
            double const d = x[size_t(r) * IN + c] - mu;
            s2 += d * d;
        }
        double const sd = std::sqrt(s2 / n);
        m->x_mean[c] = float(mu);
        m->x_inv_std[c] = sd > 1e-12 ? float(1.0 / sd) : 1.f;
        stats[c] = m->x_mean[c];
        stats[128 + c] = m->x_inv_std[c];
    }
    double s = 0, s2 = 0;
    for (uint32_t r = 0; r < n; ++r) s += y[r];
    double const mu = s / n;
    for (uint32_t r = 0; r < n; ++r) s2 += (y[r] - mu) * (y[r] - mu);
    m->y_mean = float(mu);
    m->y_std = s2 > 0 ? float(std::sqrt(s2 / n)) : 1.f;
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_stats, stats.data(), 256 * 4, cudaMemcpyHostToDevice, m->stream), "stats");
    if (upload_rows(m, x, n)) return 1;
    std::vector<float> ys(n);
    for (uint32_t r = 0; r < n; ++r) ys[r] = (y[r] - m->y_mean) / m->y_std;
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_y, ys.data(), size_t(n) * 4, cudaMemcpyHostToDevice, m->stream), "targets");
    TA3S_CUDA(m, cudaStreamSynchronize(m->stream), "set data");
    m->rows = n;
    return 0;
}

int ta3s_set_data_standardized(ta3s_model* m, const float* x, const float* y, uint32_t n) {
    if (!m || !x || !y || n == 0) return fail(m, "ta3s_set_data_standardized: need n > 0 rows");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    std::vector<float> stats(256, 0.f);
    for (int c = 0; c < 128; ++c) stats[128 + c] = 1.f;
    std::fill(m->x_mean.begin(), m->x_mean.end(), 0.f);
    std::fill(m->x_inv_std.begin(), m->x_inv_std.end(), 1.f);
    m->y_mean = 0.f;
    m->y_std = 1.f;
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_stats, stats.data(), 256 * 4, cudaMemcpyHostToDevice, m->stream), "stats");
    if (upload_rows(m, x, n)) return 1;
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_y, y, size_t(n) * 4, cudaMemcpyHostToDevice, m->stream), "targets");
    TA3S_CUDA(m, cudaStreamSynchronize(m->stream), "set data");
    m->rows = n;
    return 0;
}

int ta3s_gradients(ta3s_model* m, float* grad_out, float* loss_out) {
    if (!m || !grad_out) return fail(m, "ta3s_gradients: null argument");
    if (m->rows == 0) return fail(m, "ta3s_gradients: no data");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    TA3S_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    if (launch_mlp(m, int(m->rows), nullptr, 1)) return 1;
    if (check_status(m)) return 1;
    int const grid = std::min(int((m->rows + ROWS - 1) / ROWS), m->sms);
    std::vector<float> part(size_t(grid) * PARTIAL);
    TA3S_CUDA(m, cudaMemcpy(part.data(), m->d_partial, part.size() * 4, cudaMemcpyDeviceToHost), "partials");
    for (int i = 0; i < PARTIAL; ++i) {
        float s = 0.f;
        for (int k = 0; k < grid; ++k) s += part[size_t(k) * PARTIAL + i];
        if (i < NPARAM)
            grad_out[i] = s;
        else if (i == NPARAM && loss_out)
            *loss_out = s;
    }
    return 0;
}

int ta3s_train(ta3s_model* m, uint32_t epochs, uint32_t batch, float lr, float weight_decay, uint32_t seed,
               float* final_loss) {
    if (!m || batch == 0) return fail(m, "ta3s_train: batch must be positive");
    if (m->rows == 0) return fail(m, "ta3s_train: no data");
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    uint32_t const n = m->rows;
    uint32_t const steps_per_epoch = (n + batch - 1) / batch;
    size_t const total = size_t(epochs) * steps_per_epoch * batch;
    std::vector<int32_t> idx(total);
    std::mt19937 rng(seed);
    std::vector<int32_t> perm(n);
    for (uint32_t e = 0; e < epochs; ++e) {
        std::iota(perm.begin(), perm.end(), 0);
        std::shuffle(perm.begin(), perm.end(), rng);
        for (uint32_t s = 0; s < steps_per_epoch; ++s)
            for (uint32_t b = 0; b < batch; ++b) {
                uint32_t const k = s * batch + b;
                idx[(size_t(e) * steps_per_epoch + s) * batch + b] = k < n ? perm[k] : -1;
            }
    }
    if (grow(m, m->d_idx, m->cap_idx, std::max<size_t>(total, 1), "alloc indices")) return 1;
    TA3S_CUDA(m, cudaMemcpyAsync(m->d_idx, idx.data(), total * 4, cudaMemcpyHostToDevice, m->stream), "indices");
    TA3S_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (uint32_t e = 0; e < epochs; ++e)
        for (uint32_t s = 0; s < steps_per_epoch; ++s) {
            uint32_t const rows_here = std::min(batch, n - s * batch);
            if (launch_mlp(m, int(rows_here), m->d_idx + (size_t(e) * steps_per_epoch + s) * batch, 1)) return 1;
            ++m->adam_t;
            float const c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
            int const grid = std::min(int((rows_here + ROWS - 1) / ROWS), m->sms);
            adam_kernel<<<(PARTIAL + 255) / 256, 256, 0, m->stream>>>(m->d_param, m->d_m, m->d_v, m->d_partial, grid,
                                                                      lr, b1, b2, eps, c1, c2, weight_decay,
                                                                      m->d_w1b, m->d_w2b,
                                                                      m->d_loss);
            TA3S_CUDA(m, cudaGetLastError(), "adam launch");
        }
    if (check_status(m)) return 1;
    if (final_loss) {
        float l[2];
        TA3S_CUDA(m, cudaMemcpy(l, m->d_loss, 8, cudaMemcpyDeviceToHost), "loss");
        *final_loss = l[1] > 0 ? l[0] / l[1] : 0.f;
    }
    return 0;
}

int ta3s_predict(ta3s_model* m, const float* x, uint32_t n, float* mean_out, float* logvar_out) {
    if (!m || !x || !mean_out) return fail(m, "ta3s_predict: null argument");
    if (n == 0) return 0;
    TA3S_CUDA(m, cudaSetDevice(m->device), "set device");
    if (upload_rows(m, x, n)) return 1;
    TA3S_CUDA(m, cudaMemsetAsync(m->d_status, 0, 4, m->stream), "status");
    if (launch_mlp(m, int(n), nullptr, 0)) return 1;
    std::vector<float> out(size_t(n) * 2);
    TA3S_CUDA(m, cudaMemcpyAsync(out.data(), m->d_out, out.size() * 4, cudaMemcpyDeviceToHost, m->stream), "outputs");
    if (check_status(m)) return 1;
    for (uint32_t r = 0; r < n; ++r) {
        mean_out[r] = out[2 * r] * m->y_std + m->y_mean;
        if (logvar_out) logvar_out[r] = out[2 * r + 1] + 2.f * std::log(m->y_std);
    }
    m->rows = 0;   // the training rows were overwritten: a later train call needs set_data again
    return 0;
}

} // extern "C"
