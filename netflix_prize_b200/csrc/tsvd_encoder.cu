// Learned warm start: an amortised user encoder that predicts a user's
// factors (p_u, b_u, alpha_u) from the user's rating history, to initialise
// fold-in of new users instead of the standard init (p_u ~ N(0, sigma_u),
// b_u = alpha_u = 0). There is no counterpart in the reference; the fold-in
// itself is the reference's user-side SGD with item tables frozen
// (src/tsvdx4p.rs:390-639).
//
//   h0 = mean over the user's training ratings (i, r, t) of
//        E_item[i, r] + E_rating[r - 1] + E_date[time_bin(t)]       (dim 128)
// E_item has one row per (item, rating) pair, so h0 carries which items the
// user rated how, not only which items and which ratings.
//   h1 = GELU(h0 W1 + b1)   128 -> 512
//   h2 = GELU(h1 W2 + b2)   512 -> 512
//   y  = h2 W3 + b3         512 -> f + 2   (standardised p_u, b_u, alpha_u)
//
// Loss: mean squared error against the standardised targets. Weights are FP32
// masters with BF16 copies; every GEMM runs on the tensor cores with BF16
// operands and an FP32 accumulator in tensor memory (tcgen05.mma, 128x64
// tiles, operands brought by TMA), activations are stored as BF16 for the next GEMM and as FP32
// pre-activations for the GELU derivative. AdamW updates all parameters
// (weight decay on the matrices).
#include <cuda.h>  // CUtensorMap and the tensor-map encoder (reached through the runtime's driver entry point)
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rand_stream.hpp"
#include "tsvd_epoch.cuh"

using tsvd::Error;

namespace tsvd {
namespace {

constexpr int kEmb = 128, kHid = 512, kMaxBatch = 4096;

// ---------------------------------------------------------------------------
// C[M,N] = op(A)[M,K] . op(B)[K,N] with BF16 operands, FP32 accumulation.
// A is [M,K] row-major (a_km = 0) or stored as [K,M] (a_km = 1); B is stored
// as [K,N] (b_kn = 1) or [N,K] (b_kn = 0).
// Epilogue: + bias[n] (optional); out_f32 and/or out_bf16 (optional); with
// gelu, out_f32 receives the pre-activation and out_bf16 GELU of it.
// ---------------------------------------------------------------------------
struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K, lda, ldb, a_km, b_kn;
    const float* bias;
    float* out_f32;
    __nv_bfloat16* out_bf16;
    int ldc, gelu;
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// ---------------------------------------------------------------------------
// The register-staged GEMM (k_gemm_tc; k_gemm_tma below is the TMA-fed form
// that gemm() prefers) runs on the 5th-generation tensor cores (tcgen05): a
// 128x64 output tile per CTA with its FP32 accumulator in tensor memory. Each 64-deep K block
// of A and B is staged in shared memory as BF16 in the K-major, unswizzled
// core-matrix layout (a core matrix is 8 rows x 16 bytes; core matrices are
// 128 B apart along K and 1024 B apart along M or N). Two stages: while one
// thread's four tcgen05.mma (M = 128, N = 64, K = 16) run on one stage, all
// threads fill the other; each stage's MMAs are committed to its own mbarrier,
// which is waited on (with an iteration limit) before the stage is refilled.
// The epilogue reads the accumulator back with tcgen05.ld, one row per thread.
// ---------------------------------------------------------------------------
constexpr int TC_M = 128, TC_N = 64, TC_K = 64;
constexpr uint32_t kTcABytes = TC_M * TC_K * 2;        // 16 KB A tile per stage
constexpr uint32_t kTcBBytes = TC_N * TC_K * 2;        // 8 KB B tile per stage
constexpr uint32_t kTcStage = kTcABytes + kTcBBytes;
constexpr uint32_t kTcLBO = 128;                       // core matrices adjacent along K
constexpr uint32_t kTcSBO = (TC_K / 8) * 128;          // core matrices adjacent along M / N
constexpr uint32_t kTcSmem = 56 * 1024;                // 2 stages + mbarriers + TMEM address; caps residency
                                                       // at 4 CTAs per SM, whose 4 x 64 TMEM columns always fit
constexpr unsigned kTcWaitLimit = 1u << 20;
// instruction descriptor: D FP32, A and B BF16, both K-major, N = 64, M = 128
constexpr uint32_t kTcIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row r, k) of a staged tile
__device__ __forceinline__ uint32_t tc_off(int r, int k) {
    return (uint32_t)(r >> 3) * kTcSBO + (uint32_t)(k >> 3) * kTcLBO + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

// shared-memory matrix descriptor: start address, leading (K) and stride (M/N)
// byte offsets in 16-byte units, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((kTcLBO >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((kTcSBO >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase) {
    for (unsigned it = 0; it < kTcWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{.reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p;}"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Fill a (ROWS x TC_K) tile with rows r0.. and k0.. of X (zero outside), X
// stored [rows][K] (x_km = 0) or [K][rows] (x_km = 1); 16-byte loads along
// X's contiguous dimension where the layout allows.
template <int ROWS>
__device__ __forceinline__ void tc_stage(const __nv_bfloat16* X, int x_km, int ld, int rows, int K, int r0, int k0,
                                         uint8_t* tile, int tid) {
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    const bool vec = (ld & 7) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
    if (vec && !x_km) {
        // 8 consecutive k of one row = one core-matrix row (16 bytes)
        for (int e = tid; e < ROWS * (TC_K / 8); e += 128) {
            const int r = e / (TC_K / 8), k8 = (e % (TC_K / 8)) * 8;
            const int gr = r0 + r, gk = k0 + k8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (gr < rows) {
                if (gk + 8 <= K) {
                    v = __ldg(reinterpret_cast<const uint4*>(X + (size_t)gr * ld + gk));
                } else {
                    __nv_bfloat16 t[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) t[q] = gk + q < K ? X[(size_t)gr * ld + gk + q] : zero;
                    v = *reinterpret_cast<const uint4*>(t);
                }
            }
            *reinterpret_cast<uint4*>(tile + tc_off(r, k8)) = v;
        }
    } else if (vec) {
        // 8 consecutive rows at one k: one column of a core matrix
        for (int e = tid; e < (ROWS / 8) * TC_K; e += 128) {
            const int r8 = (e % (ROWS / 8)) * 8, k = e / (ROWS / 8);
            const int gr = r0 + r8, gk = k0 + k;
            __nv_bfloat16 t[8];
            if (gk < K && gr + 8 <= rows) {
                *reinterpret_cast<uint4*>(t) = __ldg(reinterpret_cast<const uint4*>(X + (size_t)gk * ld + gr));
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) t[q] = (gk < K && gr + q < rows) ? X[(size_t)gk * ld + gr + q] : zero;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(r8 + q, k)) = t[q];
        }
    } else {
        for (int e = tid; e < ROWS * TC_K; e += 128) {
            // consecutive threads take consecutive rows when X is stored [K][rows]
            const int r = x_km ? e % ROWS : e / TC_K, k = x_km ? e / ROWS : e % TC_K;
            const int gr = r0 + r, gk = k0 + k;
            __nv_bfloat16 v = zero;
            if (gr < rows && gk < K) v = x_km ? X[(size_t)gk * ld + gr] : X[(size_t)gr * ld + gk];
            *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(r, k)) = v;
        }
    }
}

// Register staging of one (ROWS x TC_K) operand tile: tc_load issues every
// 16-byte global load of the tile at once (so their latencies overlap each
// other and the tensor core's work on the previous block), tc_store writes
// them into the core-matrix layout. Requires 16-byte aligned rows (`vec` in
// tc_stage); element-wise fallbacks stay in tc_stage.
template <int ROWS>
struct TileRegs {
    static constexpr int N = ROWS * TC_K / 8 / 128;  // 16-byte chunks per thread
    uint4 v[N];
};

template <int ROWS>
__device__ __forceinline__ void tc_load(const __nv_bfloat16* X, int x_km, int ld, int rows, int K, int r0, int k0,
                                        TileRegs<ROWS>& t, int tid) {
#pragma unroll
    for (int c = 0; c < TileRegs<ROWS>::N; ++c) {
        const int e = tid + 128 * c;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (!x_km) {
            // 8 consecutive k of one row
            const int r = e / (TC_K / 8), k8 = (e % (TC_K / 8)) * 8;
            const int gr = r0 + r, gk = k0 + k8;
            if (gr < rows) {
                if (gk + 8 <= K) {
                    v = __ldg(reinterpret_cast<const uint4*>(X + (size_t)gr * ld + gk));
                } else {
                    __nv_bfloat16 tt[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) tt[q] = gk + q < K ? X[(size_t)gr * ld + gk + q] : __float2bfloat16(0.0f);
                    v = *reinterpret_cast<const uint4*>(tt);
                }
            }
        } else {
            // 8 consecutive rows at one k
            const int r8 = (e % (ROWS / 8)) * 8, k = e / (ROWS / 8);
            const int gr = r0 + r8, gk = k0 + k;
            if (gk < K) {
                if (gr + 8 <= rows) {
                    v = __ldg(reinterpret_cast<const uint4*>(X + (size_t)gk * ld + gr));
                } else {
                    __nv_bfloat16 tt[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        tt[q] = gr + q < rows ? X[(size_t)gk * ld + gr + q] : __float2bfloat16(0.0f);
                    v = *reinterpret_cast<const uint4*>(tt);
                }
            }
        }
        t.v[c] = v;
    }
}

template <int ROWS>
__device__ __forceinline__ void tc_store(int x_km, const TileRegs<ROWS>& t, uint8_t* tile, int tid) {
#pragma unroll
    for (int c = 0; c < TileRegs<ROWS>::N; ++c) {
        const int e = tid + 128 * c;
        if (!x_km) {
            const int r = e / (TC_K / 8), k8 = (e % (TC_K / 8)) * 8;
            *reinterpret_cast<uint4*>(tile + tc_off(r, k8)) = t.v[c];
        } else {
            const int r8 = (e % (ROWS / 8)) * 8, k = e / (ROWS / 8);
            const __nv_bfloat16* tt = reinterpret_cast<const __nv_bfloat16*>(&t.v[c]);
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(r8 + q, k)) = tt[q];
        }
    }
}

__global__ void __launch_bounds__(128) k_gemm_tc(GemmArgs g, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) uint8_t tsm[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + 2 * kTcStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tsm + 2 * kTcStage + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;
    const uint32_t s_base = smem_u32(tsm), mb0 = smem_u32(mbar), mb1 = mb0 + 8;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // split K: block z takes K blocks kb0 .. kb0 + nk - 1 (the host sizes
    // gridDim.z so that none is empty) and writes its partial tile to slice z
    const int nk_all = (g.K + TC_K - 1) / TC_K;
    const int per = (nk_all + (int)gridDim.z - 1) / (int)gridDim.z;
    const int kb0 = (int)blockIdx.z * per;
    const int nk = min(nk_all, kb0 + per) - kb0;
    float* const out_f32 = g.out_f32 ? g.out_f32 + (size_t)blockIdx.z * g.M * g.ldc : nullptr;
    // 16-byte rows on both operands: register-staged pipeline (the next
    // block's loads in flight during this block's MMAs); else element-wise
    const bool vec_a = (g.lda & 7) == 0 && (reinterpret_cast<uintptr_t>(g.A) & 15) == 0;
    const bool vec_b = (g.ldb & 7) == 0 && (reinterpret_cast<uintptr_t>(g.B) & 15) == 0;
    const bool piped = vec_a && vec_b;
    TileRegs<TC_M> ra;
    TileRegs<TC_N> rb;
    if (piped) {
        tc_load<TC_M>(g.A, g.a_km, g.lda, g.M, g.K, m0, kb0 * TC_K, ra, tid);
        tc_load<TC_N>(g.B, g.b_kn, g.ldb, g.N, g.K, n0, kb0 * TC_K, rb, tid);
        tc_store<TC_M>(g.a_km, ra, tsm, tid);
        tc_store<TC_N>(g.b_kn, rb, tsm + kTcABytes, tid);
    } else {
        tc_stage<TC_M>(g.A, g.a_km, g.lda, g.M, g.K, m0, kb0 * TC_K, tsm, tid);
        tc_stage<TC_N>(g.B, g.b_kn, g.ldb, g.N, g.K, n0, kb0 * TC_K, tsm + kTcABytes, tid);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    for (int kb = 0; kb < nk && ok; ++kb) {
        const uint32_t st = (uint32_t)(kb & 1);
        if (tid == 0) {
            const uint32_t a_s = s_base + st * kTcStage, b_s = a_s + kTcABytes;
#pragma unroll
            for (int kk = 0; kk < TC_K / 16; ++kk) {
                const uint64_t ad = tc_desc(a_s + (uint32_t)kk * 2u * kTcLBO);
                const uint64_t bd = tc_desc(b_s + (uint32_t)kk * 2u * kTcLBO);
                const uint32_t accumulate = (kb > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{.reg .pred p; setp.ne.u32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;}" ::"r"(
                        tmem),
                    "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             st ? mb1 : mb0)
                         : "memory");
        }
        if (kb + 1 < nk) {
            if (piped) {
                // the next block's loads go out before the wait for the other stage
                tc_load<TC_M>(g.A, g.a_km, g.lda, g.M, g.K, m0, (kb0 + kb + 1) * TC_K, ra, tid);
                tc_load<TC_N>(g.B, g.b_kn, g.ldb, g.N, g.K, n0, (kb0 + kb + 1) * TC_K, rb, tid);
            }
            // the other stage was read by block kb - 1's MMAs
            if (kb >= 1) {
                const uint32_t ps = (uint32_t)((kb - 1) & 1), par = (uint32_t)(((kb - 1) >> 1) & 1);
                ok = __syncthreads_and(tc_wait(ps ? mb1 : mb0, par) ? 1 : 0) != 0;
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;");
            }
            uint8_t* nxt = tsm + (st ^ 1u) * kTcStage;
            if (piped) {
                tc_store<TC_M>(g.a_km, ra, nxt, tid);
                tc_store<TC_N>(g.b_kn, rb, nxt + kTcABytes, tid);
            } else {
                tc_stage<TC_M>(g.A, g.a_km, g.lda, g.M, g.K, m0, (kb0 + kb + 1) * TC_K, nxt, tid);
                tc_stage<TC_N>(g.B, g.b_kn, g.ldb, g.N, g.K, n0, (kb0 + kb + 1) * TC_K, nxt + kTcABytes, tid);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;");
        }
    }
    if (ok) {
        // the last commit covers every MMA issued before it
        const uint32_t ls = (uint32_t)((nk - 1) & 1), par = (uint32_t)(((nk - 1) >> 1) & 1);
        ok = __syncthreads_and(tc_wait(ls ? mb1 : mb0, par) ? 1 : 0) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1u);
        const uint32_t ls = (uint32_t)((nk - 1) & 1), par = (uint32_t)(((nk - 1) >> 1) & 1);
        tc_wait(ls ? mb1 : mb0, par);  // one more bounded wait for the MMAs in flight
    } else {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < TC_N; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= g.N) continue;
                    float x = __uint_as_float(v[j]);
                    if (g.bias) x += g.bias[n];
                    if (out_f32) out_f32[(size_t)m * g.ldc + n] = x;
                    if (g.out_bf16) g.out_bf16[(size_t)m * g.ldc + n] = __float2bfloat16(g.gelu ? gelu_f(x) : x);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_N));
}

// Sum of the split-K slices ws[z] (z = 0 .. splits-1, in that order) into out.
__global__ void k_splitk_sum(const float* __restrict__ ws, int splits, int M, int N, int ldc, float* __restrict__ out) {
    const size_t total = (size_t)M * N;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t at = (e / N) * ldc + e % N;
        float acc = ws[at];
        for (int z = 1; z < splits; ++z) acc += ws[(size_t)z * M * ldc + at];
        out[at] = acc;
    }
}

// ---------------------------------------------------------------------------
// TMA-fed GEMM (k_gemm_tma) for K-major operands with 16-byte aligned rows
// (gemm() transposes MN-major operands into a workspace first). Each K block
// of A (128 rows) and B (64 rows) arrives as eight cp.async.bulk.tensor 2-D
// tile loads of 8 K-columns x all rows of the tile (16 bytes per row): box g
// lands at g x ROWS x 16 bytes, which is the K-major no-swizzle core-matrix
// layout with K-adjacent core matrices ROWS x 16 bytes apart (LBO) and M- or
// N-adjacent ones 128 bytes apart (SBO). The tensor maps' bounds give the zero
// fill past M, N and K. kTmaStages stages: thread 0 issues a stage's loads
// once the MMAs of its previous use have committed (the stage's empty
// barrier); thread 32 issues the stage's four MMAs (M = 128, N = 64, K = 16)
// once its loads have landed (full barrier, transaction bytes) and commits
// them to the empty barrier; the last commit releases the epilogue. Every wait
// is bounded; a wait that gives up sets *err and the kernel carries on, so all
// issued work drains before the block exits. No multicast.
// ---------------------------------------------------------------------------
constexpr int kTmaStages = 4;
constexpr uint32_t kTmaSmem = kTmaStages * kTcStage + 128;  // stages, 2 x kTmaStages + 1 mbarriers, TMEM address
constexpr uint32_t kTmaLboA = TC_M * 16, kTmaLboB = TC_N * 16, kTmaSbo = 128;

__device__ __forceinline__ uint64_t tma_desc(uint32_t addr, uint32_t lbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((kTmaSbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tma_tile(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(mbar)
        : "memory");
}

__global__ void __launch_bounds__(128) k_gemm_tma(const __grid_constant__ CUtensorMap tmA,
                                                  const __grid_constant__ CUtensorMap tmB, GemmArgs g,
                                                  unsigned* __restrict__ err) {
    extern __shared__ __align__(16) uint8_t tsm[];
    uint64_t* full = reinterpret_cast<uint64_t*>(tsm + kTmaStages * kTcStage);
    uint64_t* empty = full + kTmaStages;
    uint64_t* done = empty + kTmaStages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;
    const uint32_t s_base = smem_u32(tsm);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2 * kTmaStages + 1; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + b)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // split K as in k_gemm_tc: block z takes K blocks kb0 .. kb0 + nk - 1
    const int nk_all = (g.K + TC_K - 1) / TC_K;
    const int per = (nk_all + (int)gridDim.z - 1) / (int)gridDim.z;
    const int kb0 = (int)blockIdx.z * per;
    const int nk = min(nk_all, kb0 + per) - kb0;
    float* const out_f32 = g.out_f32 ? g.out_f32 + (size_t)blockIdx.z * g.M * g.ldc : nullptr;
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    if (tid == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
        for (int kb = 0; kb < nk; ++kb) {
            const int st = kb % kTmaStages, use = kb / kTmaStages;
            if (use > 0 && !tc_wait(smem_u32(empty + st), (uint32_t)((use - 1) & 1))) atomicOr(err, 1u);
            const uint32_t fb = smem_u32(full + st);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(kTcStage) : "memory");
            const uint32_t a_s = s_base + (uint32_t)st * kTcStage, b_s = a_s + kTcABytes;
            const int k0 = (kb0 + kb) * TC_K;
#pragma unroll
            for (int g8 = 0; g8 < TC_K / 8; ++g8) {
                tma_tile(a_s + (uint32_t)g8 * kTmaLboA, &tmA, k0 + 8 * g8, m0, fb);
                tma_tile(b_s + (uint32_t)g8 * kTmaLboB, &tmB, k0 + 8 * g8, n0, fb);
            }
        }
    } else if (tid == 32) {
        for (int kb = 0; kb < nk; ++kb) {
            const int st = kb % kTmaStages, use = kb / kTmaStages;
            if (!tc_wait(smem_u32(full + st), (uint32_t)(use & 1))) atomicOr(err, 1u);
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a_s = s_base + (uint32_t)st * kTcStage, b_s = a_s + kTcABytes;
#pragma unroll
            for (int kk = 0; kk < TC_K / 16; ++kk) {
                const uint64_t ad = tma_desc(a_s + (uint32_t)kk * 2u * kTmaLboA, kTmaLboA);
                const uint64_t bd = tma_desc(b_s + (uint32_t)kk * 2u * kTmaLboB, kTmaLboB);
                const uint32_t accumulate = (kb > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{.reg .pred p; setp.ne.u32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;}" ::"r"(
                        tmem),
                    "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(empty + st))
                         : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(done))
                     : "memory");
    }
    __syncwarp();
    const bool ok = __syncthreads_and(tc_wait(smem_u32(done), 0u) ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok) {
        if (tid == 0) atomicOr(err, 1u);
    } else {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < TC_N; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= g.N) continue;
                    float x = __uint_as_float(v[j]);
                    if (g.bias) x += g.bias[n];
                    if (out_f32) out_f32[(size_t)m * g.ldc + n] = x;
                    if (g.out_bf16) g.out_bf16[(size_t)m * g.ldc + n] = __float2bfloat16(g.gelu ? gelu_f(x) : x);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_N));
}

// out[c][r] = in[r][c] (r < R, c < C); in has leading dimension ld_in, out ld_out.
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C, int ld_in,
                                 __nv_bfloat16* __restrict__ out, int ld_out) {
    __shared__ __nv_bfloat16 t[32][34];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        if (r < R && c < C) t[y][threadIdx.x] = in[(size_t)r * ld_in + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (c < C && r < R) out[(size_t)c * ld_out + r] = t[threadIdx.x][y];
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Tensor map of a K-major BF16 operand X[rows][K] (leading dimension ld, a
// multiple of 8; 16-byte aligned base): boxes of 8 K-columns x box_rows rows.
bool k_major_map(CUtensorMap* map, const __nv_bfloat16* X, int K, int rows, int ld, int box_rows) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {8u, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1u, 1u};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(X), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// `err` receives 1 when an MMA completion wait ran out (the results are then invalid).
// splits > 1 (FP32 output only, no bias or activation) divides K over that many
// blocks per tile, through ws (splits * M * ldc floats), summed in a fixed order.
// tws (tws_elems BF16 elements) takes the transposed copies of MN-major
// operands for the TMA path; without room there, or with operands whose rows
// are not 16-byte aligned, the register-staged kernel runs instead.
void gemm(cudaStream_t st, unsigned* err, const __nv_bfloat16* A, int a_km, int lda, const __nv_bfloat16* B, int b_kn, int ldb, int M,
          int N, int K, const float* bias, float* out_f32, __nv_bfloat16* out_bf16, int ldc, int gelu, int splits = 1,
          float* ws = nullptr, __nv_bfloat16* tws = nullptr, size_t tws_elems = 0) {
    // K = 0 would issue no MMA and leave the accumulator uninitialised
    if (M <= 0 || N <= 0 || K <= 0) throw Error(TSVD_ERR_INVALID, "gemm: M, N and K must be positive");
    const int nk = (K + TC_K - 1) / TC_K;
    splits = std::max(1, std::min(splits, nk));
    if (splits > 1) {
        const int per = (nk + splits - 1) / splits;
        splits = (nk + per - 1) / per;  // no empty slice
    }
    const bool split = splits > 1 && ws && out_f32 && !bias && !out_bf16 && !gelu;
    if (!split) splits = 1;
    dim3 grid((N + TC_N - 1) / TC_N, (M + TC_M - 1) / TC_M, splits);
    // TMA path: every operand K-major with 16-byte aligned rows, MN-major ones
    // transposed into tws first (leading dimension K rounded up to 8)
    const int k8 = (K + 7) & ~7;
    const size_t need = (a_km ? (size_t)M * k8 : 0) + (b_kn ? (size_t)N * k8 : 0);
    bool tma = encode_tiled() != nullptr && need <= (tws ? tws_elems : 0);
    if (!a_km && ((lda & 7) || (reinterpret_cast<uintptr_t>(A) & 15))) tma = false;
    if (!b_kn && ((ldb & 7) || (reinterpret_cast<uintptr_t>(B) & 15))) tma = false;
    if (tma) {
        const __nv_bfloat16* Ak = A;
        const __nv_bfloat16* Bk = B;
        int ldak = lda, ldbk = ldb;
        __nv_bfloat16* p = tws;
        const dim3 tb(32, 8);
        if (a_km) {  // A stored [K][M]
            k_transpose_bf16<<<dim3((M + 31) / 32, (K + 31) / 32), tb, 0, st>>>(A, K, M, lda, p, k8);
            TSVD_CUDA(cudaGetLastError());
            Ak = p;
            ldak = k8;
            p += (size_t)M * k8;
        }
        if (b_kn) {  // B stored [K][N]
            k_transpose_bf16<<<dim3((N + 31) / 32, (K + 31) / 32), tb, 0, st>>>(B, K, N, ldb, p, k8);
            TSVD_CUDA(cudaGetLastError());
            Bk = p;
            ldbk = k8;
        }
        CUtensorMap ma, mb;
        tma = k_major_map(&ma, Ak, K, M, ldak, TC_M) && k_major_map(&mb, Bk, K, N, ldbk, TC_N);
        if (tma) {
            GemmArgs g{Ak, Bk, M, N, K, ldak, ldbk, 0, 0, bias, split ? ws : out_f32, out_bf16, ldc, gelu};
            TSVD_CUDA(cudaFuncSetAttribute(k_gemm_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmem));
            k_gemm_tma<<<grid, 128, kTmaSmem, st>>>(ma, mb, g, err);
            TSVD_CUDA(cudaGetLastError());
        }
    }
    if (!tma) {
        GemmArgs g{A, B, M, N, K, lda, ldb, a_km, b_kn, bias, split ? ws : out_f32, out_bf16, ldc, gelu};
        TSVD_CUDA(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
        k_gemm_tc<<<grid, 128, kTcSmem, st>>>(g, err);
        TSVD_CUDA(cudaGetLastError());
    }
    if (split) {
        k_splitk_sum<<<(unsigned)std::min<size_t>(((size_t)M * N + 255) / 256, 148 * 8), 256, 0, st>>>(ws, splits, M, N, ldc,
                                                                                                    out_f32);
        TSVD_CUDA(cudaGetLastError());
    }
}

// ---------------------------------------------------------------------------
// Embedding bag over a batch of users, one block per user: the 8 warps take
// the user's 32-rating chunks in turn (8 rows in flight per warp) and sum the
// (item, rating) rows; the rating and date-bin rows enter through the user's
// histograms, hist[w] = {counts of ratings 1..5, counts of date bins}, which
// the block also writes for the backward pass. Partial sums are combined in
// warp order, so results do not depend on scheduling.
// ---------------------------------------------------------------------------
constexpr int kBagWarps = 8;

__global__ void __launch_bounds__(kBagWarps * 32) k_embag_fwd(DeviceState s, const int8_t* __restrict__ raw,
                                                            const uint32_t* __restrict__ users, int n,
                                                            const float* __restrict__ e_item,
                                                            const float* __restrict__ e_rate,
                                                            const float* __restrict__ e_date, float* __restrict__ h0,
                                                            __nv_bfloat16* __restrict__ h0b, float* __restrict__ hist,
                                                            float* __restrict__ inv_n) {
    __shared__ float4 part[kBagWarps][32];
    __shared__ int cnt_sh[5 + kMaxBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int w = blockIdx.x;
    const uint32_t T = s.T, H = 5 + T;
    for (uint32_t k = threadIdx.x; k < H; k += blockDim.x) cnt_sh[k] = 0;
    __syncthreads();
    const uint32_t u = users[w];
    const uint64_t a = s.user_off[u], b = s.user_off[u + 1];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint64_t base = a + (uint64_t)warp * 32; base < b; base += (uint64_t)kBagWarps * 32) {
        const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
        uint32_t row = 0;
        if ((uint32_t)lane < cnt) {
            const Rec r = load_rec(s.rec + base + lane);
            const int rt = min(max((int)raw[base + lane], 1), 5) - 1;
            row = rec_id(r.key) * 5u + (uint32_t)rt;
            atomicAdd(&cnt_sh[rt], 1);
            atomicAdd(&cnt_sh[5 + rec_tbin(r.key)], 1);
        }
        for (uint32_t j = 0; j < cnt; j += 8) {
            float4 x[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t ro = __shfl_sync(kFull, row, (int)(j + q < cnt ? j + q : j));
                x[q] = __ldg(reinterpret_cast<const float4*>(e_item + (size_t)ro * kEmb) + lane);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                if (j + q < cnt) {
                    acc.x += x[q].x; acc.y += x[q].y; acc.z += x[q].z; acc.w += x[q].w;
                }
            }
        }
    }
    part[warp][lane] = acc;
    __syncthreads();
    if (warp == 0) {
        float4 t = part[0][lane];
#pragma unroll
        for (int k = 1; k < kBagWarps; ++k) {
            const float4 v = part[k][lane];
            t.x += v.x; t.y += v.y; t.z += v.z; t.w += v.w;
        }
        for (uint32_t k = 0; k < H; ++k) {
            const float c = (float)cnt_sh[k];
            if (c == 0.0f) continue;
            const float* tab = k < 5 ? e_rate + (size_t)k * kEmb : e_date + (size_t)(k - 5) * kEmb;
            const float4 v = __ldg(reinterpret_cast<const float4*>(tab) + lane);
            t.x += c * v.x; t.y += c * v.y; t.z += c * v.z; t.w += c * v.w;
        }
        const float inv = b > a ? 1.0f / (float)(b - a) : 0.0f;
        t.x *= inv; t.y *= inv; t.z *= inv; t.w *= inv;
        reinterpret_cast<float4*>(h0 + (size_t)w * kEmb)[lane] = t;
        __nv_bfloat16* o = h0b + (size_t)w * kEmb + 4 * lane;
        o[0] = __float2bfloat16(t.x); o[1] = __float2bfloat16(t.y);
        o[2] = __float2bfloat16(t.z); o[3] = __float2bfloat16(t.w);
        if (lane == 0) inv_n[w] = inv;
    }
    for (uint32_t k = threadIdx.x; k < H; k += blockDim.x) hist[(size_t)w * H + k] = (float)cnt_sh[k];
}

// dE_item[i, r] += dh0 / n_u for every rating of the user (vector atomics:
// users share items); one block per user, warps as in the forward pass.
__global__ void __launch_bounds__(kBagWarps * 32) k_embag_bwd(DeviceState s, const int8_t* __restrict__ raw,
                                                            const uint32_t* __restrict__ users, int n,
                                                            const float* __restrict__ dh0,
                                                            const float* __restrict__ inv_n,
                                                            float* __restrict__ g_item) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int w = blockIdx.x;
    const uint32_t u = users[w];
    const uint64_t a = s.user_off[u], b = s.user_off[u + 1];
    if (a == b) return;
    const float inv = inv_n[w];
    float4 d = reinterpret_cast<const float4*>(dh0 + (size_t)w * kEmb)[lane];
    d.x *= inv; d.y *= inv; d.z *= inv; d.w *= inv;
    for (uint64_t base = a + (uint64_t)warp * 32; base < b; base += (uint64_t)kBagWarps * 32) {
        const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
        uint32_t row = 0;
        if ((uint32_t)lane < cnt) {
            const Rec r = load_rec(s.rec + base + lane);
            row = rec_id(r.key) * 5u + (uint32_t)(min(max((int)raw[base + lane], 1), 5) - 1);
        }
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t ro = __shfl_sync(kFull, row, (int)j);
            float* gi = g_item + (size_t)ro * kEmb + 4 * lane;
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(gi), "f"(d.x), "f"(d.y), "f"(d.z),
                         "f"(d.w)
                         : "memory");
        }
    }
}

// Gradients of the rating and date-bin rows from the histograms:
// g[k][c] = sum over the batch, in order, of hist[w][k] * dh0[w][c] / n_w
// (k < 5: rating rows, else date-bin rows). One block per row k.
__global__ void __launch_bounds__(kEmb) k_hist_grad(const float* __restrict__ hist, uint32_t H,
                                                    const float* __restrict__ dh0, const float* __restrict__ inv_n,
                                                    int n, float* __restrict__ g_rate, float* __restrict__ g_date) {
    const uint32_t k = blockIdx.x, c = threadIdx.x;
    float acc = 0.0f;
    int w = 0;
    for (; w + 4 <= n; w += 4) {
        float h[4], d[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            h[q] = __ldg(hist + (size_t)(w + q) * H + k) * __ldg(inv_n + w + q);
            d[q] = __ldg(dh0 + (size_t)(w + q) * kEmb + c);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) acc += h[q] * d[q];
    }
    for (; w < n; ++w) acc += __ldg(hist + (size_t)w * H + k) * __ldg(inv_n + w) * __ldg(dh0 + (size_t)w * kEmb + c);
    if (k < 5) g_rate[(size_t)k * kEmb + c] = acc;
    else g_date[(size_t)(k - 5) * kEmb + c] = acc;
}

// Standardised targets of a batch: [p_u (f), b_u, alpha_u].
__global__ void k_targets(DeviceState s, const uint32_t* __restrict__ users, int n, int O,
                          const float* __restrict__ mean, const float* __restrict__ inv_std, float* __restrict__ t) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * O) return;
    const int r = e / O, c = e % O;
    const uint32_t u = users[r];
    float v;
    if (c < (int)s.F) v = s.ufeat[(size_t)u * s.Fs + c];
    else if (c == (int)s.F) v = s.ubias[u];
    else v = s.alpha_u[u];
    t[e] = (v - mean[c]) * inv_std[c];
}

// dY = 2 (y - t) / (n * O); per-block partial sums of the squared error.
// dyb is stored with leading dimension ldb >= O (16-byte rows for the GEMM's
// vector staging).
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, int total, int O, int ldb,
                      float scale, float* __restrict__ dy, __nv_bfloat16* __restrict__ dyb,
                      double* __restrict__ part) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const float d = y[e] - t[e];
        acc += (double)d * d;
        const float g = 2.0f * d * scale;
        dy[e] = g;
        dyb[(size_t)(e / O) * ldb + e % O] = __float2bfloat16(g);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dZ = dH * GELU'(Z) -> BF16
__global__ void k_gelu_bwd(const float* __restrict__ dh, const float* __restrict__ z, int total,
                           __nv_bfloat16* __restrict__ dzb) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x)
        dzb[e] = __float2bfloat16(dh[e] * gelu_grad(z[e]));
}

// column sums of a [rows, cols] matrix (bias gradients)
// Column sums out[c] = sum_r x[r][c] (x [rows][cols]) in two fixed-order
// levels, so that many blocks share the rows and the result does not depend on
// scheduling: block (bx, by) sums rows by * kColRows .. of columns 32 bx ..
// with 8 row lanes (rows r, r + 8, ... each) and adds the lanes in order into
// part[by][c]; k_colsum_fin adds the row chunks in order.
constexpr int kColRows = 256;

template <class T>
__device__ __forceinline__ float as_float(T v);
template <>
__device__ __forceinline__ float as_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ float as_float<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <class T>
__global__ void k_colsum_part(const T* __restrict__ x, int rows, int cols, float* __restrict__ part) {
    __shared__ float sh[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int r0 = blockIdx.y * kColRows, r1 = min(rows, r0 + kColRows);
    float a = 0.0f;
    if (c < cols)
        for (int r = r0 + (int)threadIdx.y; r < r1; r += 8) a += as_float<T>(x[(size_t)r * cols + c]);
    sh[threadIdx.y][threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.0f;
#pragma unroll
        for (int y = 0; y < 8; ++y) t += sh[y][threadIdx.x];
        part[(size_t)blockIdx.y * cols + c] = t;
    }
}

__global__ void k_colsum_fin(const float* __restrict__ part, int chunks, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float a = 0.0f;
    for (int k = 0; k < chunks; ++k) a += part[(size_t)k * cols + c];
    out[c] = a;
}

// out = column sums of x [rows][cols] through the workspace part
// (ceil(rows / kColRows) * cols floats)
template <class T>
void colsum(cudaStream_t st, const T* x, int rows, int cols, float* part, float* out) {
    const int chunks = (rows + kColRows - 1) / kColRows;
    k_colsum_part<T><<<dim3((cols + 31) / 32, chunks), dim3(32, 8), 0, st>>>(x, rows, cols, part);
    k_colsum_fin<<<(cols + 127) / 128, 128, 0, st>>>(part, chunks, cols, out);
    TSVD_CUDA(cudaGetLastError());
}

// The batch's mean squared error sse / count from the k_mse block partials
// (added in block order), into loss[0]; with `acc`, also added to the epoch's
// running sum loss[1].
__global__ void k_loss(const double* __restrict__ part, int nb, double count, double* __restrict__ loss, int acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sse = 0.0;
    for (int b = 0; b < nb; ++b) sse += part[b];
    loss[0] = sse / count;
    if (acc) loss[1] += loss[0];
}

__global__ void k_adamw(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                        float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float wd, float c1,
                        float c2, __nv_bfloat16* __restrict__ wb, uint32_t cols, uint32_t ldb) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float gg = g[e];
        const float mm = b1 * m[e] + (1.0f - b1) * gg;
        const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        const float upd = (mm / c1) / (sqrtf(vv / c2) + eps) + wd * w[e];
        const float nw = w[e] - lr * upd;
        w[e] = nw;
        if (wb) wb[(e / cols) * ldb + e % cols] = __float2bfloat16(nw);
    }
}

// y keeps x's rows of `cols` values at leading dimension ldb
__global__ void k_f32_to_bf16(const float* __restrict__ x, size_t n, __nv_bfloat16* __restrict__ y, uint32_t cols,
                              uint32_t ldb) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        y[(e / cols) * ldb + e % cols] = __float2bfloat16(x[e]);
}

// Writes de-standardised predictions into the model's user tables and resets
// the rest of each user's state to the standard init (p2 = 0, but_bin = 0,
// cu = 1, ubias_day = 0 on the user's days).
__global__ void k_apply_users(DeviceState s, const uint32_t* __restrict__ users, int n, int O,
                              const float* __restrict__ y, const float* __restrict__ mean,
                              const float* __restrict__ std) {
    const int w = blockIdx.x;
    if (w >= n) return;
    const uint32_t u = users[w];
    for (uint32_t c = threadIdx.x; c < s.Fs; c += blockDim.x) {
        s.ufeat[(size_t)u * s.Fs + c] = c < s.F ? y[(size_t)w * O + c] * std[c] + mean[c] : 0.0f;
        s.ufeat2[(size_t)u * s.Fs + c] = 0.0f;
    }
    for (uint32_t b = threadIdx.x; b < s.T; b += blockDim.x) s.but_bin[(size_t)u * s.T + b] = 0.0f;
    for (uint64_t d = s.ud_start[u] + threadIdx.x; d < s.ud_start[u + 1]; d += blockDim.x) s.ubias_day[d] = 0.0f;
    if (threadIdx.x == 0) {
        s.ubias[u] = y[(size_t)w * O + s.F] * std[s.F] + mean[s.F];
        s.alpha_u[u] = y[(size_t)w * O + s.F + 1] * std[s.F + 1] + mean[s.F + 1];
        s.cu[u] = 1.0f;
    }
}

struct Param {
    std::string name;
    size_t n;
    bool decay;
    uint32_t cols = 1, ldb = 1;  // row length and BF16 leading dimension (a multiple of 8) of wb
    DevMem w, g, m, v, wb;       // wb only for GEMM weights
};

}  // namespace
}  // namespace tsvd

struct tsvd_encoder {
    const tsvd_model* model = nullptr;
    int O = 0;
    int Op = 0;  // O rounded up to a multiple of 8: leading dimension of the BF16 copies of W3 and dY
    float lr = 1e-3f, wd = 1e-4f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    uint64_t step = 0;
    std::vector<tsvd::Param> params;  // e_item, e_rate, e_date, W1, b1, W2, b2, W3, b3
    tsvd::DevMem raw, mean, inv_std, std_;
    tsvd::DevMem users, h0, h0b, z1, h1b, z2, h2b, y, t, dy, dyb, dh2, dz2b, dh1, dz1b, dh0, part;
    tsvd::DevMem hist, inv_n;  // per batch user: rating and date-bin counts, 1 / history length
    tsvd::DevMem loss;         // {the last batch's loss, the epoch's sum of batch losses} (FP64)
    tsvd::DevMem epoch_users;  // the users of a training epoch, device copy
    tsvd::DevMem tc_err;       // set by the tensor-core GEMM when an MMA wait ran out
    tsvd::DevMem ws;           // split-K partial tiles of the weight-gradient GEMMs
    tsvd::DevMem tws;          // transposed copies of MN-major GEMM operands (TMA path)
    size_t tws_elems = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string err;
    double last_loss = 0.0;
};

namespace {

thread_local std::string g_enc_err;

tsvd::Param& P(tsvd_encoder* e, int k) { return e->params[k]; }

template <class F>
int eguard(tsvd_encoder* e, F&& f) {
    try {
        f();
        return TSVD_OK;
    } catch (const Error& x) {
        if (e) e->err = x.what();
        g_enc_err = x.what();
        return x.status;
    } catch (const std::exception& x) {
        if (e) e->err = x.what();
        g_enc_err = x.what();
        return TSVD_ERR_INVALID;
    }
}

unsigned grid_for(size_t n, unsigned block = 256) {
    return (unsigned)std::min<size_t>((n + block - 1) / block, 148 * 32);
}

// forward over n users already in e->users; fills y (and activations)
void forward(tsvd_encoder* e, int n) {
    using namespace tsvd;
    const DeviceState& s = e->model->d;
    cudaStream_t st = e->stream;
    k_embag_fwd<<<n, kBagWarps * 32, 0, st>>>(s, e->raw.as<int8_t>(), e->users.as<uint32_t>(), n,
                                              P(e, 0).w.as<float>(), P(e, 1).w.as<float>(), P(e, 2).w.as<float>(),
                                              e->h0.as<float>(), e->h0b.as<__nv_bfloat16>(), e->hist.as<float>(),
                                              e->inv_n.as<float>());
    TSVD_CUDA(cudaGetLastError());
    gemm(st, e->tc_err.as<unsigned>(), e->h0b.as<__nv_bfloat16>(), 0, kEmb, P(e, 3).wb.as<__nv_bfloat16>(), 1, kHid, n, kHid, kEmb,
         P(e, 4).w.as<float>(), e->z1.as<float>(), e->h1b.as<__nv_bfloat16>(), kHid, 1, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
    gemm(st, e->tc_err.as<unsigned>(), e->h1b.as<__nv_bfloat16>(), 0, kHid, P(e, 5).wb.as<__nv_bfloat16>(), 1, kHid, n, kHid, kHid,
         P(e, 6).w.as<float>(), e->z2.as<float>(), e->h2b.as<__nv_bfloat16>(), kHid, 1, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
    gemm(st, e->tc_err.as<unsigned>(), e->h2b.as<__nv_bfloat16>(), 0, kHid, P(e, 7).wb.as<__nv_bfloat16>(), 1, e->Op, n, e->O, kHid,
         P(e, 8).w.as<float>(), e->y.as<float>(), nullptr, e->O, 0, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
}

// Gradients for n users in e->users (targets from the model). The batch's
// loss goes to e->loss[0] on the device (and is added to the epoch's sum in
// e->loss[1] with `acc`); with `read` it is also returned (one stream
// synchronisation), else 0.
double backward(tsvd_encoder* e, int n, bool read, bool acc) {
    using namespace tsvd;
    const DeviceState& s = e->model->d;
    cudaStream_t st = e->stream;
    const int O = e->O;
    k_targets<<<(n * O + 255) / 256, 256, 0, st>>>(s, e->users.as<uint32_t>(), n, O, e->mean.as<float>(),
                                                   e->inv_std.as<float>(), e->t.as<float>());
    const int nb = 256;
    const int Op = e->Op;
    k_mse<<<nb, 256, 0, st>>>(e->y.as<float>(), e->t.as<float>(), n * O, O, Op, 1.0f / ((float)n * O),
                              e->dy.as<float>(), e->dyb.as<__nv_bfloat16>(), e->part.as<double>());
    TSVD_CUDA(cudaGetLastError());
    // layer 3
    gemm(st, e->tc_err.as<unsigned>(), e->h2b.as<__nv_bfloat16>(), 1, kHid, e->dyb.as<__nv_bfloat16>(), 1, Op, kHid, O, n, nullptr,
         P(e, 7).g.as<float>(), nullptr, O, 0, 8, e->ws.as<float>(), e->tws.as<__nv_bfloat16>(), e->tws_elems);
    colsum<float>(st, e->dy.as<float>(), n, O, e->ws.as<float>(), P(e, 8).g.as<float>());
    gemm(st, e->tc_err.as<unsigned>(), e->dyb.as<__nv_bfloat16>(), 0, Op, P(e, 7).wb.as<__nv_bfloat16>(), 0, Op, n, kHid, O, nullptr,
         e->dh2.as<float>(), nullptr, kHid, 0, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
    k_gelu_bwd<<<grid_for((size_t)n * kHid), 256, 0, st>>>(e->dh2.as<float>(), e->z2.as<float>(), n * kHid,
                                                           e->dz2b.as<__nv_bfloat16>());
    // layer 2
    gemm(st, e->tc_err.as<unsigned>(), e->h1b.as<__nv_bfloat16>(), 1, kHid, e->dz2b.as<__nv_bfloat16>(), 1, kHid, kHid, kHid, n, nullptr,
         P(e, 5).g.as<float>(), nullptr, kHid, 0, 4, e->ws.as<float>(), e->tws.as<__nv_bfloat16>(), e->tws_elems);
    colsum<__nv_bfloat16>(st, e->dz2b.as<__nv_bfloat16>(), n, kHid, e->ws.as<float>(), P(e, 6).g.as<float>());
    gemm(st, e->tc_err.as<unsigned>(), e->dz2b.as<__nv_bfloat16>(), 0, kHid, P(e, 5).wb.as<__nv_bfloat16>(), 0, kHid, n, kHid, kHid, nullptr,
         e->dh1.as<float>(), nullptr, kHid, 0, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
    k_gelu_bwd<<<grid_for((size_t)n * kHid), 256, 0, st>>>(e->dh1.as<float>(), e->z1.as<float>(), n * kHid,
                                                           e->dz1b.as<__nv_bfloat16>());
    // layer 1
    gemm(st, e->tc_err.as<unsigned>(), e->h0b.as<__nv_bfloat16>(), 1, kEmb, e->dz1b.as<__nv_bfloat16>(), 1, kHid, kEmb, kHid, n, nullptr,
         P(e, 3).g.as<float>(), nullptr, kHid, 0, 16, e->ws.as<float>(), e->tws.as<__nv_bfloat16>(), e->tws_elems);
    colsum<__nv_bfloat16>(st, e->dz1b.as<__nv_bfloat16>(), n, kHid, e->ws.as<float>(), P(e, 4).g.as<float>());
    gemm(st, e->tc_err.as<unsigned>(), e->dz1b.as<__nv_bfloat16>(), 0, kHid, P(e, 3).wb.as<__nv_bfloat16>(), 0, kHid, n, kEmb, kHid, nullptr,
         e->dh0.as<float>(), nullptr, kEmb, 0, 1, nullptr, e->tws.as<__nv_bfloat16>(), e->tws_elems);
    // embeddings
    for (int k = 0; k < 3; ++k) TSVD_CUDA(cudaMemsetAsync(P(e, k).g.p, 0, P(e, k).n * 4, st));
    k_embag_bwd<<<n, kBagWarps * 32, 0, st>>>(s, e->raw.as<int8_t>(), e->users.as<uint32_t>(), n,
                                              e->dh0.as<float>(), e->inv_n.as<float>(), P(e, 0).g.as<float>());
    k_hist_grad<<<5 + s.T, kEmb, 0, st>>>(e->hist.as<float>(), 5 + s.T, e->dh0.as<float>(), e->inv_n.as<float>(), n,
                                          P(e, 1).g.as<float>(), P(e, 2).g.as<float>());
    TSVD_CUDA(cudaGetLastError());
    k_loss<<<1, 32, 0, st>>>(e->part.as<double>(), nb, (double)n * O, e->loss.as<double>(), acc ? 1 : 0);
    TSVD_CUDA(cudaGetLastError());
    if (!read) return 0.0;
    double l = 0.0;
    TSVD_CUDA(cudaMemcpyAsync(&l, e->loss.p, 8, cudaMemcpyDeviceToHost, st));
    TSVD_CUDA(cudaStreamSynchronize(st));
    return l;
}

void adamw_step(tsvd_encoder* e) {
    using namespace tsvd;
    e->step++;
    const float c1 = 1.0f - std::pow(e->b1, (float)e->step), c2 = 1.0f - std::pow(e->b2, (float)e->step);
    for (auto& p : e->params)
        k_adamw<<<grid_for(p.n), 256, 0, e->stream>>>(p.w.as<float>(), p.g.as<float>(), p.m.as<float>(),
                                                      p.v.as<float>(), p.n, e->lr, e->b1, e->b2, e->eps,
                                                      p.decay ? e->wd : 0.0f, c1, c2,
                                                      p.wb.p ? p.wb.as<__nv_bfloat16>() : nullptr, p.cols, p.ldb);
    TSVD_CUDA(cudaGetLastError());
}

// A tensor-core GEMM whose MMA wait ran out leaves its flag set: report it.
void check_tc(tsvd_encoder* e) {
    unsigned f = 0;
    TSVD_CUDA(cudaMemcpyAsync(&f, e->tc_err.p, 4, cudaMemcpyDeviceToHost, e->stream));
    TSVD_CUDA(cudaStreamSynchronize(e->stream));
    if (f) throw Error(TSVD_ERR_TIMEOUT, "encoder GEMM: a tensor-core MMA did not complete within its wait limit");
}

void set_users(tsvd_encoder* e, const uint32_t* users, int n) {
    TSVD_CUDA(cudaMemcpyAsync(e->users.p, users, (size_t)n * 4, cudaMemcpyHostToDevice, e->stream));
}

}  // namespace

extern "C" {

int tsvd_encoder_create(const tsvd_model* m, const int8_t* train_raw, const uint32_t* target_users,
                        uint64_t n_target, uint64_t seed, float lr, float weight_decay, tsvd_encoder** out) {
    if (!m || !out || !train_raw) return TSVD_ERR_INVALID;
    *out = nullptr;
    tsvd_encoder* e = new tsvd_encoder();
    int rc = eguard(e, [&] {
        using namespace tsvd;
        TSVD_CUDA(cudaSetDevice(m->device));
        e->model = m;
        e->lr = lr;
        e->wd = weight_decay;
        const DeviceState& s = m->d;
        if (s.F < 1 || s.F > 256) throw Error(TSVD_ERR_UNSUPPORTED, "the user encoder is built for n_feat in 1..256");
        e->O = (int)s.F + 2;
        e->Op = (e->O + 7) & ~7;
        TSVD_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->raw.alloc(s.n_train);
        TSVD_CUDA(cudaMemcpy(e->raw.p, train_raw, s.n_train, cudaMemcpyHostToDevice));
        // parameters: Xavier-uniform matrices, N(0, 0.05) embeddings, zero biases
        ChaCha12Stream g(seed);
        auto add = [&](const char* name, size_t n, bool decay, bool bf16, float scale, bool uniform,
                       uint32_t cols = 1) {
            Param p;
            p.name = name;
            p.n = n;
            p.decay = decay;
            p.cols = cols;
            p.ldb = (cols + 7) & ~7u;
            std::vector<float> h(n, 0.0f);
            if (scale > 0) {
                for (size_t k = 0; k < n; ++k) {
                    if (uniform) h[k] = scale * (2.0f * (float)(g.u32() >> 8) * (1.0f / 16777216.0f) - 1.0f);
                    else h[k] = scale * (float)std_normal(g);
                }
            }
            p.w.alloc(n * 4);
            TSVD_CUDA(cudaMemcpy(p.w.p, h.data(), n * 4, cudaMemcpyHostToDevice));
            p.g.alloc(n * 4);
            p.m.alloc(n * 4);
            p.v.alloc(n * 4);
            TSVD_CUDA(cudaMemset(p.m.p, 0, n * 4));
            TSVD_CUDA(cudaMemset(p.v.p, 0, n * 4));
            if (bf16) {
                const size_t nb = n / cols * p.ldb;
                p.wb.alloc(nb * 2);
                TSVD_CUDA(cudaMemset(p.wb.p, 0, nb * 2));
                k_f32_to_bf16<<<grid_for(n), 256>>>(p.w.as<float>(), n, p.wb.as<__nv_bfloat16>(), p.cols, p.ldb);
                TSVD_CUDA(cudaGetLastError());
            }
            e->params.push_back(std::move(p));
        };
        const int O = e->O;
        // (item, rating) rows, N(0, 0.05) drawn on the device from a stream of their own
        add("e_item", (size_t)s.n_items * 5 * kEmb, false, false, 0.0f, false);
        {
            const NormalTable t{e->params.back().w.as<float>(), (uint64_t)s.n_items * 5, (uint32_t)kEmb,
                                (uint32_t)kEmb, 0.05f};
            device_normal_tables(&t, 1, seed ^ 0x5eed5eed5eed5eedull, e->stream);
            TSVD_CUDA(cudaStreamSynchronize(e->stream));
        }
        add("e_rate", 5 * kEmb, false, false, 0.05f, false);
        add("e_date", (size_t)s.T * kEmb, false, false, 0.05f, false);
        add("w1", (size_t)kEmb * kHid, true, true, std::sqrt(6.0f / (kEmb + kHid)), true, kHid);
        add("b1", kHid, false, false, 0.0f, false);
        add("w2", (size_t)kHid * kHid, true, true, std::sqrt(6.0f / (kHid + kHid)), true, kHid);
        add("b2", kHid, false, false, 0.0f, false);
        add("w3", (size_t)kHid * O, true, true, std::sqrt(6.0f / (kHid + O)), true, (uint32_t)O);
        add("b3", (size_t)O, false, false, 0.0f, false);
        // target standardisation from the model's factors of the target users
        std::vector<float> mean(O, 0.0f), sd(O, 1.0f);
        if (target_users && n_target) {
            std::vector<float> uf((size_t)s.n_users * s.F), ub(s.n_users), al(s.n_users);
            TSVD_CUDA(cudaMemcpy2D(uf.data(), s.F * 4, s.ufeat, s.Fs * 4, s.F * 4, s.n_users, cudaMemcpyDeviceToHost));
            TSVD_CUDA(cudaMemcpy(ub.data(), s.ubias, s.n_users * 4, cudaMemcpyDeviceToHost));
            TSVD_CUDA(cudaMemcpy(al.data(), s.alpha_u, s.n_users * 4, cudaMemcpyDeviceToHost));
            std::vector<double> s1(O, 0.0), s2(O, 0.0);
            for (uint64_t k = 0; k < n_target; ++k) {
                const uint32_t u = target_users[k];
                if (u >= s.n_users) throw Error(TSVD_ERR_INVALID, "target user out of range");
                for (int c = 0; c < O; ++c) {
                    const double v = c < (int)s.F ? uf[(size_t)u * s.F + c] : (c == (int)s.F ? ub[u] : al[u]);
                    s1[c] += v;
                    s2[c] += v * v;
                }
            }
            for (int c = 0; c < O; ++c) {
                const double mu = s1[c] / n_target, var = std::max(s2[c] / n_target - mu * mu, 1e-20);
                mean[c] = (float)mu;
                sd[c] = (float)std::sqrt(var);
            }
        }
        std::vector<float> inv(O);
        for (int c = 0; c < O; ++c) inv[c] = 1.0f / sd[c];
        e->mean.alloc(O * 4);
        e->inv_std.alloc(O * 4);
        e->std_.alloc(O * 4);
        TSVD_CUDA(cudaMemcpy(e->mean.p, mean.data(), O * 4, cudaMemcpyHostToDevice));
        TSVD_CUDA(cudaMemcpy(e->inv_std.p, inv.data(), O * 4, cudaMemcpyHostToDevice));
        TSVD_CUDA(cudaMemcpy(e->std_.p, sd.data(), O * 4, cudaMemcpyHostToDevice));
        // activations for kMaxBatch users
        const size_t B = kMaxBatch;
        e->users.alloc(B * 4);
        e->h0.alloc(B * kEmb * 4);
        e->h0b.alloc(B * kEmb * 2);
        e->z1.alloc(B * kHid * 4);
        e->h1b.alloc(B * kHid * 2);
        e->z2.alloc(B * kHid * 4);
        e->h2b.alloc(B * kHid * 2);
        e->y.alloc(B * O * 4);
        e->t.alloc(B * O * 4);
        e->dy.alloc(B * O * 4);
        e->dyb.alloc(B * e->Op * 2);
        e->dh2.alloc(B * kHid * 4);
        e->dz2b.alloc(B * kHid * 2);
        e->dh1.alloc(B * kHid * 4);
        e->dz1b.alloc(B * kHid * 2);
        e->dh0.alloc(B * kEmb * 4);
        e->part.alloc(256 * 8);
        e->hist.alloc((size_t)B * (5 + s.T) * 4);
        e->inv_n.alloc((size_t)B * 4);
        e->tc_err.alloc(4);
        e->loss.alloc(16);
        TSVD_CUDA(cudaMemset(e->loss.p, 0, 16));
        // split-K slices: dW1 16 x 128 x 512, dW2 4 x 512 x 512, dW3 8 x 512 x O
        e->ws.alloc(std::max(std::max((size_t)16 * kEmb * kHid, (size_t)4 * kHid * kHid), (size_t)8 * kHid * O) * 4);
        // two transposed operands of at most 512 rows x max(batch, 512) columns
        e->tws_elems = (size_t)2 * kHid * std::max(kMaxBatch, kHid);
        e->tws.alloc(e->tws_elems * 2);
        TSVD_CUDA(cudaMemset(e->tc_err.p, 0, 4));
        TSVD_CUDA(cudaDeviceSynchronize());
    });
    if (rc != TSVD_OK) {
        tsvd_encoder_destroy(e);
        return rc;
    }
    *out = e;
    return TSVD_OK;
}

void tsvd_encoder_destroy(tsvd_encoder* e) {
    if (!e) return;
    if (e->stream) {
        cudaStreamSynchronize(e->stream);
        cudaStreamDestroy(e->stream);
    }
    delete e;
}

// One pass over `users` in mini-batches (batch <= 4096): forward, loss,
// backward, AdamW. Returns the mean loss over the pass.
int tsvd_encoder_train_epoch(tsvd_encoder* e, const uint32_t* users, uint64_t n, uint32_t batch, double* mean_loss) {
    if (!e || !users) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        if (batch == 0 || batch > (uint32_t)tsvd::kMaxBatch) throw Error(TSVD_ERR_INVALID, "batch must be 1..4096");
        TSVD_CUDA(cudaSetDevice(e->model->device));
        for (uint64_t k = 0; k < n; ++k)
            if (users[k] >= e->model->d.n_users) throw Error(TSVD_ERR_INVALID, "user out of range");
        // the batches' users go up once; the batch losses are summed on the
        // device, so the epoch runs without a host round trip per batch
        if (e->epoch_users.bytes < n * 4) e->epoch_users.alloc(n * 4);
        TSVD_CUDA(cudaMemcpyAsync(e->epoch_users.p, users, n * 4, cudaMemcpyHostToDevice, e->stream));
        TSVD_CUDA(cudaMemsetAsync(e->loss.p, 0, 16, e->stream));
        uint64_t nb = 0;
        for (uint64_t a = 0; a < n; a += batch) {
            const int b = (int)std::min<uint64_t>(batch, n - a);
            TSVD_CUDA(cudaMemcpyAsync(e->users.p, e->epoch_users.as<uint32_t>() + a, (size_t)b * 4,
                                      cudaMemcpyDeviceToDevice, e->stream));
            forward(e, b);
            backward(e, b, false, true);
            adamw_step(e);
            nb++;
        }
        double sums[2] = {0.0, 0.0};
        TSVD_CUDA(cudaMemcpyAsync(sums, e->loss.p, 16, cudaMemcpyDeviceToHost, e->stream));
        TSVD_CUDA(cudaStreamSynchronize(e->stream));
        check_tc(e);
        e->last_loss = nb ? sums[1] / nb : 0.0;
        if (mean_loss) *mean_loss = e->last_loss;
    });
}

// Loss and gradients for one batch without an update (for checking); the
// gradients are read with tsvd_encoder_get("g.<name>").
int tsvd_encoder_loss_grad(tsvd_encoder* e, const uint32_t* users, uint32_t n, double* loss) {
    if (!e || !users) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        if (n == 0 || n > (uint32_t)tsvd::kMaxBatch) throw Error(TSVD_ERR_INVALID, "n must be 1..4096");
        TSVD_CUDA(cudaSetDevice(e->model->device));
        set_users(e, users, (int)n);
        forward(e, (int)n);
        const double l = backward(e, (int)n, true, false);
        check_tc(e);
        if (loss) *loss = l;
    });
}

// Standardised outputs y [n, f+2] for `users` (host copy).
int tsvd_encoder_forward(tsvd_encoder* e, const uint32_t* users, uint32_t n, float* out) {
    if (!e || !users || !out) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        if (n == 0 || n > (uint32_t)tsvd::kMaxBatch) throw Error(TSVD_ERR_INVALID, "n must be 1..4096");
        TSVD_CUDA(cudaSetDevice(e->model->device));
        set_users(e, users, (int)n);
        forward(e, (int)n);
        TSVD_CUDA(cudaMemcpyAsync(out, e->y.p, (size_t)n * e->O * 4, cudaMemcpyDeviceToHost, e->stream));
        TSVD_CUDA(cudaStreamSynchronize(e->stream));
        check_tc(e);
    });
}

// Writes the encoder's prediction of p_u, b_u, alpha_u into model m (which
// may be e's model) for `users`; their other user state is reset to the
// standard init.
int tsvd_encoder_apply(tsvd_encoder* e, tsvd_model* m, const uint32_t* users, uint64_t n) {
    if (!e || !m || !users) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        using namespace tsvd;
        if (m->d.F != e->model->d.F || m->d.n_users != e->model->d.n_users)
            throw Error(TSVD_ERR_INVALID, "model shape differs from the encoder's");
        TSVD_CUDA(cudaSetDevice(e->model->device));
        for (uint64_t a = 0; a < n; a += kMaxBatch) {
            const int b = (int)std::min<uint64_t>(kMaxBatch, n - a);
            for (int k = 0; k < b; ++k)
                if (users[a + k] >= m->d.n_users) throw Error(TSVD_ERR_INVALID, "user out of range");
            set_users(e, users + a, b);
            forward(e, b);
            k_apply_users<<<b, 128, 0, e->stream>>>(m->d, e->users.as<uint32_t>(), b, e->O, e->y.as<float>(),
                                                    e->mean.as<float>(), e->std_.as<float>());
            TSVD_CUDA(cudaGetLastError());
        }
        TSVD_CUDA(cudaStreamSynchronize(e->stream));
        check_tc(e);
    });
}

// Parameter (or gradient, "g.<name>") access: names e_item, e_rate, e_date,
// w1, b1, w2, b2, w3, b3; FP32 row-major, matrices [in, out].
int tsvd_encoder_get(const tsvd_encoder* ec, const char* name, float* dst, uint64_t count) {
    tsvd_encoder* e = const_cast<tsvd_encoder*>(ec);
    if (!e || !name || !dst) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        std::string n(name);
        bool grad = n.rfind("g.", 0) == 0;
        if (grad) n = n.substr(2);
        for (auto& p : e->params)
            if (p.name == n) {
                if (count != p.n) throw Error(TSVD_ERR_INVALID, "count mismatch for " + n);
                TSVD_CUDA(cudaMemcpy(dst, grad ? p.g.p : p.w.p, count * 4, cudaMemcpyDeviceToHost));
                return;
            }
        throw Error(TSVD_ERR_INVALID, "unknown encoder parameter " + n);
    });
}

int tsvd_encoder_set(tsvd_encoder* e, const char* name, const float* src, uint64_t count) {
    if (!e || !name || !src) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(e->mu);
    return eguard(e, [&] {
        using namespace tsvd;
        for (auto& p : e->params)
            if (p.name == name) {
                if (count != p.n) throw Error(TSVD_ERR_INVALID, "count mismatch");
                TSVD_CUDA(cudaMemcpy(p.w.p, src, count * 4, cudaMemcpyHostToDevice));
                if (p.wb.p) {
                    k_f32_to_bf16<<<grid_for(p.n), 256, 0, e->stream>>>(p.w.as<float>(), p.n,
                                                                       p.wb.as<__nv_bfloat16>(), p.cols, p.ldb);
                    TSVD_CUDA(cudaStreamSynchronize(e->stream));
                }
                return;
            }
        throw Error(TSVD_ERR_INVALID, std::string("unknown encoder parameter ") + name);
    });
}

// Standardisation used for the targets: mean[f+2], std[f+2].
int tsvd_encoder_target_stats(const tsvd_encoder* ec, float* mean, float* std_out) {
    tsvd_encoder* e = const_cast<tsvd_encoder*>(ec);
    if (!e || !mean || !std_out) return TSVD_ERR_INVALID;
    return eguard(e, [&] {
        TSVD_CUDA(cudaMemcpy(mean, e->mean.p, e->O * 4, cudaMemcpyDeviceToHost));
        TSVD_CUDA(cudaMemcpy(std_out, e->std_.p, e->O * 4, cudaMemcpyDeviceToHost));
    });
}

const char* tsvd_encoder_last_error(const tsvd_encoder* e) { return e ? e->err.c_str() : g_enc_err.c_str(); }

}  // extern "C"
