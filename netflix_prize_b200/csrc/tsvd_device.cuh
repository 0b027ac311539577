// Device-side helpers shared by the tsvdx4 kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsvd_model.hpp"

namespace tsvd {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// A feature row of Fs = 32 * VPL floats is spread over a warp, VPL values per
// lane. Element of (lane, slot): for VPL % 4 == 0 each lane owns float4 runs
// (128-float stripes), for VPL == 2 a float2, otherwise one float per
// 32-float stripe. Every layout makes a warp-wide row access fully coalesced.
template <int VPL>
struct Row {
    __device__ __forceinline__ static int elem(int lane, int v) {
        if constexpr (VPL % 4 == 0) return (v >> 2) * 128 + (lane << 2) + (v & 3);
        else if constexpr (VPL == 2) return (lane << 1) + v;
        else return v * 32 + lane;
    }
    // L2-coherent load (bypasses L1): rows that other warps may update.
    __device__ __forceinline__ static void load_cg(const float* row, int lane, float (&x)[VPL]) {
        if constexpr (VPL % 4 == 0) {
#pragma unroll
            for (int c = 0; c < VPL / 4; ++c) {
                float4 t = __ldcg(reinterpret_cast<const float4*>(row + c * 128 + lane * 4));
                x[4 * c] = t.x; x[4 * c + 1] = t.y; x[4 * c + 2] = t.z; x[4 * c + 3] = t.w;
            }
        } else if constexpr (VPL == 2) {
            float2 t = __ldcg(reinterpret_cast<const float2*>(row + lane * 2));
            x[0] = t.x; x[1] = t.y;
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) x[v] = __ldcg(row + v * 32 + lane);
        }
    }
    // Read-only path: rows that no thread writes during the kernel.
    __device__ __forceinline__ static void load_nc(const float* row, int lane, float (&x)[VPL]) {
        if constexpr (VPL % 4 == 0) {
#pragma unroll
            for (int c = 0; c < VPL / 4; ++c) {
                float4 t = __ldg(reinterpret_cast<const float4*>(row + c * 128 + lane * 4));
                x[4 * c] = t.x; x[4 * c + 1] = t.y; x[4 * c + 2] = t.z; x[4 * c + 3] = t.w;
            }
        } else if constexpr (VPL == 2) {
            float2 t = __ldg(reinterpret_cast<const float2*>(row + lane * 2));
            x[0] = t.x; x[1] = t.y;
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) x[v] = __ldg(row + v * 32 + lane);
        }
    }
    __device__ __forceinline__ static void store(float* row, int lane, const float (&x)[VPL]) {
        if constexpr (VPL % 4 == 0) {
#pragma unroll
            for (int c = 0; c < VPL / 4; ++c)
                __stcg(reinterpret_cast<float4*>(row + c * 128 + lane * 4),
                       make_float4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]));
        } else if constexpr (VPL == 2) {
            __stcg(reinterpret_cast<float2*>(row + lane * 2), make_float2(x[0], x[1]));
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) __stcg(row + v * 32 + lane, x[v]);
        }
    }
    // Element-wise atomic add of a row delta (vector reductions where the
    // layout allows).
    __device__ __forceinline__ static void red_add(float* row, int lane, const float (&x)[VPL]) {
        if constexpr (VPL % 4 == 0) {
#pragma unroll
            for (int c = 0; c < VPL / 4; ++c) {
                float* a = row + c * 128 + lane * 4;
                asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(a), "f"(x[4 * c]),
                             "f"(x[4 * c + 1]), "f"(x[4 * c + 2]), "f"(x[4 * c + 3])
                             : "memory");
            }
        } else if constexpr (VPL == 2) {
            float* a = row + lane * 2;
            asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(a), "f"(x[0]), "f"(x[1]) : "memory");
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) atomicAdd(row + v * 32 + lane, x[v]);
        }
    }
};

__device__ __forceinline__ uint32_t rec_id(uint32_t key) { return key & kIdMask; }
__device__ __forceinline__ uint32_t rec_tbin(uint32_t key) { return (key >> 20) & 63u; }
__device__ __forceinline__ uint32_t rec_fbin(uint32_t key) { return key >> 26; }

__device__ __forceinline__ Rec load_rec(const Rec* p) {
    int4 v = __ldg(reinterpret_cast<const int4*>(p));
    Rec r;
    r.key = (uint32_t)v.x;
    r.res = __int_as_float(v.y);
    r.dev = __int_as_float(v.z);
    r.ud = (uint32_t)v.w;
    return r;
}

__device__ __forceinline__ Rec shfl_rec(const Rec& r, int src) {
    Rec o;
    o.key = __shfl_sync(kFull, r.key, src);
    o.res = __shfl_sync(kFull, r.res, src);
    o.dev = __shfl_sync(kFull, r.dev, src);
    o.ud = __shfl_sync(kFull, r.ud, src);
    return o;
}

// time_bin (src/tx.rs:285-290)
__device__ __forceinline__ uint32_t time_bin(int32_t day, int32_t day_range, uint32_t T) {
    int64_t b = ((int64_t)day * (int64_t)T) / (int64_t)day_range;
    if (b < 0) b = 0;  // dates are non-negative in every dataset; guard the cast
    return b > (int64_t)(T - 1) ? T - 1 : (uint32_t)b;
}

// dev_u(t) = sign(dt) |dt|^beta with dt = day - tu_mean[u] (src/tx.rs:292-300)
__device__ __forceinline__ float dev_of(int32_t day, float tu_mean, float beta) {
    float dt = (float)day - tu_mean;
    if (dt == 0.0f) return 0.0f;
    float s = dt > 0.0f ? 1.0f : -1.0f;
    return s * powf(fabsf(dt), beta);
}

// OrdinalHead (src/lib.rs:500-609): P(Y <= k) = sigmoid(th[k-1] - score).
__device__ __forceinline__ float sigmoid_f(float x) { return 1.0f / (1.0f + expf(-x)); }

// d(-log P(Y = y)) / d(score), y in 1..5 (OrdinalHead::grad, src/lib.rs:562-598)
__device__ __forceinline__ float ordinal_grad(const float (&th)[4], float score, int y) {
    float f[6], a[6];
    f[0] = 0.0f;
    f[5] = 1.0f;
#pragma unroll
    for (int k = 1; k < 5; ++k) f[k] = sigmoid_f(th[k - 1] - score);
#pragma unroll
    for (int k = 0; k < 6; ++k) a[k] = f[k] * (1.0f - f[k]);
    float fy = f[1], fy1 = f[0], ay = a[1], ay1 = a[0];
#pragma unroll
    for (int k = 2; k <= 5; ++k)
        if (y == k) {
            fy = f[k];
            fy1 = f[k - 1];
            ay = a[k];
            ay1 = a[k - 1];
        }
    const float p_y = fmaxf(fy - fy1, 1e-6f);
    return (ay - ay1) / p_y;
}

// E[r] = sum_k k P(Y = k) (TxModel::predict with the head, src/tx.rs:716-722)
__device__ __forceinline__ float ordinal_expect(const float* th, float score) {
    float f[6];
    f[0] = 0.0f;
    f[5] = 1.0f;
#pragma unroll
    for (int k = 1; k < 5; ++k) f[k] = sigmoid_f(th[k - 1] - score);
    return 1.0f * (f[1] - f[0]) + 2.0f * (f[2] - f[1]) + 3.0f * (f[3] - f[2]) + 4.0f * (f[4] - f[3]) +
           5.0f * (f[5] - f[4]);
}

// freq_bin (src/tx.rs:87-90)
__device__ __forceinline__ uint32_t freq_bin(uint32_t day_cnt, uint32_t NF) {
    if (day_cnt <= 1) return 0;
    float v = floorf(log2f((float)day_cnt));
    float cap = (float)(NF - 1);
    return (uint32_t)fminf(v, cap);
}

// SparseUD::index (src/tx.rs:76-83): binary search of the user's sorted days.
// Returns 0xffffffff when absent.
__device__ __forceinline__ uint32_t ud_index(const DeviceState& s, uint32_t u, int16_t day) {
    uint64_t lo = s.ud_start[u], hi = s.ud_start[u + 1];
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        int16_t d = s.ud_date[mid];
        if (d < day) lo = mid + 1;
        else hi = mid;
    }
    if (lo < s.ud_start[u + 1] && s.ud_date[lo] == day) return (uint32_t)lo;
    return 0xffffffffu;
}

}  // namespace tsvd

namespace tsvd {

// ---- asynchronous global -> shared copies (cp.async); each lane copies and
// later reads only its own elements, so a lane's own wait_group suffices.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy this lane's elements of a feature row into a shared-memory row with the
// same layout, and read them back.
template <int VPL>
__device__ __forceinline__ void row_cp_async(float* srow, const float* grow, int lane) {
    if constexpr (VPL % 4 == 0) {
#pragma unroll
        for (int c = 0; c < VPL / 4; ++c) cp_async16(srow + c * 128 + lane * 4, grow + c * 128 + lane * 4);
    } else if constexpr (VPL == 2) {
        cp_async8(srow + lane * 2, grow + lane * 2);
    } else {
#pragma unroll
        for (int v = 0; v < VPL; ++v) cp_async4(srow + v * 32 + lane, grow + v * 32 + lane);
    }
}

template <int VPL>
__device__ __forceinline__ void row_from_smem(const float* srow, int lane, float (&x)[VPL]) {
    if constexpr (VPL % 4 == 0) {
#pragma unroll
        for (int c = 0; c < VPL / 4; ++c) {
            const float4 t = *reinterpret_cast<const float4*>(srow + c * 128 + lane * 4);
            x[4 * c] = t.x; x[4 * c + 1] = t.y; x[4 * c + 2] = t.z; x[4 * c + 3] = t.w;
        }
    } else if constexpr (VPL == 2) {
        const float2 t = *reinterpret_cast<const float2*>(srow + lane * 2);
        x[0] = t.x; x[1] = t.y;
    } else {
#pragma unroll
        for (int v = 0; v < VPL; ++v) x[v] = srow[v * 32 + lane];
    }
}

}  // namespace tsvd
