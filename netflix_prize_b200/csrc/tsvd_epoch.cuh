// Declarations shared by the epoch translation units (tsvd_epoch.cu: Hogwild
// pass, ycache rebuild, epoch driver; tsvd_strat.cu: stratified schedule).
#pragma once
#include <cuda_bf16.h>

#include "tsvd_device.cuh"

namespace tsvd {

constexpr int kWarps = 8;  // warps per block
constexpr int kThreads = kWarps * 32;
// Hogwild ring slot: q row, q^f row, then kSlotScalars floats of item-side
// scalars (a multiple of 4, so every row stays 16-byte aligned). After the
// slots, a window of kRecWindow rating records (16 bytes each).
constexpr uint32_t kSlotScalars = 4;
constexpr uint32_t kRecWindow = 64;

// Shared-memory floats of one warp's Hogwild ring with `st` slots.
__host__ __device__ __forceinline__ uint32_t hog_ring_floats(int st, uint32_t Fs) {
    return (uint32_t)st * (2 * Fs + kSlotScalars) + kRecWindow * 4;
}

struct EpochParams {
    float lr_u, lr_u2, lr_ub, lr_ubd, lr_i, lr_ib, lr_y, lr_yb, lr_tu, lr_ti, lr_ta, lr_ibf, lr_iqf, lr_cu;
    float reg_iqf, reg_cu, reg_u, reg_u2, reg_i, reg_y;
    float lr_ud, reg_ud, lr_yd, reg_yd;  // per-day terms (low_memory = false)
    float lr_t, reg_t;                   // ordinal-head thresholds (sequential schedule)
    int32_t has_ud;                      // ufeat_day trained: !low_memory && lr_ud != 0
    float w_bias, w_factor;
    float nsvd_norm_exp;
    int32_t sum_err_bug;
    int32_t full_su;
    int32_t use_ycache;  // su of a user equals ycache[u] (stratified, full_su, ycache valid)
    int32_t stages;      // Hogwild prefetch ring depth (2..4) in the batched form
};

// Batched Hogwild epoch over (variant, user) units and the batched rebuild
// (tsvd_epoch.cu); states/params are device arrays, one entry per variant.
void launch_hog_batched(cudaStream_t st, const DeviceState* d_states, const EpochParams* d_params,
                        const uint32_t* d_units, uint32_t n_units, uint32_t ring_floats, uint32_t* d_counter);
void launch_rebuild_batched(cudaStream_t st, const DeviceState* d_states, uint32_t n_models, uint32_t n_users);

EpochParams make_params(const tsvd_model* m);

constexpr int kBatch = 8;  // feature rows in flight in the y gathers and updates

// su += y_j (and sub += b_j when yb is given) for the items item_of(0..n-1)
// of table y, added in order, kBatch rows in flight.
template <int VPL, class ItemOf>
__device__ __forceinline__ void gather_rows8(const float* y_tab, const float* yb_tab, uint32_t Fs, uint64_t n,
                                             ItemOf item_of, int lane, float (&su)[VPL], float& sub) {
    for (uint64_t base = 0; base < n; base += 32) {
        const uint32_t cnt = (uint32_t)(n - base < 32 ? n - base : 32);
        const uint32_t mine = lane < (int)cnt ? item_of(base + lane) : 0u;
        for (uint32_t j = 0; j < cnt; j += kBatch) {
            float y[kBatch][VPL], yb[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const uint32_t it = __shfl_sync(kFull, mine, j + q < cnt ? j + q : cnt - 1);
                Row<VPL>::load_cg(y_tab + (size_t)it * Fs, lane, y[q]);
                yb[q] = yb_tab ? __ldcg(yb_tab + it) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                if (j + q < cnt) {
#pragma unroll
                    for (int v = 0; v < VPL; ++v) su[v] += y[q][v];
                    sub += yb[q];
                }
            }
        }
    }
}

// su += y_j, sub += b_j over the NSVD1 table y (yfeat, ybias).
template <int VPL, class ItemOf>
__device__ __forceinline__ void gather_y8(const DeviceState& s, uint64_t n, ItemOf item_of, int lane,
                                          float (&su)[VPL], float& sub) {
    gather_rows8<VPL>(s.yfeat, s.ybias, s.Fs, n, item_of, lane, su, sub);
}

// BF16 read copies of FP32 master rows (same padded layout, 2 bytes/element).
struct Bf16Copies {
    const __nv_bfloat16* ifeat;   // [I, Fs]
    const __nv_bfloat16* qf0;     // [I, Fs] frequency-bin-0 rows of ifeat_freq
    const __nv_bfloat16* yfeat;   // [I, Fs]
    const __nv_bfloat16* pyc;     // [U, Fs] p_u + ycache_u
    const __nv_bfloat16* ufeat2;  // [U, Fs]
};

// Element (lane, v) of a bf16 row in Row<VPL>'s layout, widened to FP32.
template <int VPL>
__device__ __forceinline__ void row_load_bf16(const __nv_bfloat16* row, int lane, float (&x)[VPL]) {
    if constexpr (VPL % 4 == 0) {
#pragma unroll
        for (int c = 0; c < VPL / 4; ++c) {
            const uint2 t = __ldg(reinterpret_cast<const uint2*>(row + c * 128 + lane * 4));
            const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t.x));
            const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t.y));
            x[4 * c] = a.x; x[4 * c + 1] = a.y; x[4 * c + 2] = b.x; x[4 * c + 3] = b.y;
        }
    } else if constexpr (VPL == 2) {
        const unsigned t = __ldg(reinterpret_cast<const unsigned*>(row + lane * 2));
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t));
        x[0] = a.x; x[1] = a.y;
    } else {
#pragma unroll
        for (int v = 0; v < VPL; ++v) x[v] = __bfloat162float(row[v * 32 + lane]);
    }
}

#define TSVD_DISPATCH(VPLV, CALL)                                              \
    switch (VPLV) {                                                            \
        case 1: { constexpr int V = 1; CALL; } break;                          \
        case 2: { constexpr int V = 2; CALL; } break;                          \
        case 3: { constexpr int V = 3; CALL; } break;                          \
        case 4: { constexpr int V = 4; CALL; } break;                          \
        case 5: { constexpr int V = 5; CALL; } break;                          \
        case 6: { constexpr int V = 6; CALL; } break;                          \
        case 7: { constexpr int V = 7; CALL; } break;                          \
        case 8: { constexpr int V = 8; CALL; } break;                          \
        default: throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256");       \
    }

template <class K>
unsigned persistent_grid(K kernel, size_t smem) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return (unsigned)(sms * per_sm);
}

// tsvd_strat.cu
void stratified_epoch(tsvd_model* m, const EpochParams& p);
// tsvd_epoch.cu
// pyc (optional, [U, Fs]) receives p_u + ycache_u for every user
void launch_rebuild_ycache(tsvd_model* m, float* pyc = nullptr);

}  // namespace tsvd
