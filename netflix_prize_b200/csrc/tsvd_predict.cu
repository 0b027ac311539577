// Batched prediction: TxModel::predict (src/tx.rs:713-724 via factor_parts
// :303-339), predict_subscores (:651-711), and the FP64 sum of squared errors
// behind calc_rmse (src/lib.rs:659-672). One warp per row; the SSE is reduced
// in a fixed order (per-warp sums, per-block tree, then one block over the
// block partials), so repeated calls are bitwise identical.
#include <algorithm>
#include <mutex>
#include <string>

#include "tsvd_device.cuh"

namespace tsvd {
namespace {

constexpr int kWarps = 8, kThreads = 256;
constexpr unsigned kSseBlocks = 148 * 4;

struct PredParams {
    float beta;
    int32_t low_memory;
    int32_t ordinal;  // apply the ordinal head: E[r] from the cumulative logits
};

// predict (src/tx.rs:713-724): score, or E[r] under the ordinal head
__device__ __forceinline__ float finish_score(const DeviceState& s, const PredParams& pp, float bp, float dot) {
    const float score = bp + dot + 0.0f;
    return pp.ordinal ? ordinal_expect(s.thresholds, score) : score;
}

template <int VPL>
__device__ __forceinline__ void predict_row(const DeviceState& s, const PredParams& pp, uint32_t u, uint32_t i,
                                            int16_t day, int lane, float& bias_part, float& dot, float* subs) {
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    const uint32_t b = time_bin(day, s.day_range, T);
    const float dv = dev_of(day, s.tu_mean[u], pp.beta);
    const uint32_t idx = ud_index(s, u, day);
    const bool has = idx != 0xffffffffu;
    const uint32_t f = has ? freq_bin(s.ud_cnt[idx], NF) : 0u;
    const float bu_day = has ? s.ubias_day[idx] : 0.0f;
    const float ubu = s.ubias[u], but = s.but_bin[(size_t)u * T + b], al = s.alpha_u[u], ycb = s.ycache_bias[u];
    const float ibi = s.ibias[i], bit = s.bit_bin[(size_t)i * T + b], ibf = s.ibias_freq[(size_t)i * NF + f];
    const float bu_t = ubu + but + al * dv + bu_day + ycb;
    const float bi_t = ibi + bit + ibf;
    const float cu_t = s.cu[u] + (has ? s.cut[idx] : 0.0f);
    // per-day terms, low_memory = false (src/tx.rs:329-334, :692-699)
    const bool per_day = !pp.low_memory && has;
    // rows wider than 32 * VPL columns (n_feat > 256) are taken in slices of
    // 32 * VPL columns; each element's arithmetic is the same
    float part = 0.0f, mf = 0.0f, ns = 0.0f;
    for (uint32_t c0 = 0; c0 < Fs; c0 += 32 * VPL) {
        float pu[VPL], p2[VPL], su[VPL], q[VPL], qf[VPL];
        Row<VPL>::load_nc(s.ufeat + (size_t)u * Fs + c0, lane, pu);
        Row<VPL>::load_nc(s.ufeat2 + (size_t)u * Fs + c0, lane, p2);
        Row<VPL>::load_nc(s.ycache + (size_t)u * Fs + c0, lane, su);
        Row<VPL>::load_nc(s.ifeat + (size_t)i * Fs + c0, lane, q);
        Row<VPL>::load_nc(s.ifeat_freq + ((size_t)i * NF + f) * Fs + c0, lane, qf);
        float pd[VPL], sd[VPL];
        if (per_day) {
            Row<VPL>::load_nc(s.ufeat_day + (size_t)idx * Fs + c0, lane, pd);
            Row<VPL>::load_nc(s.ycache_day + (size_t)idx * Fs + c0, lane, sd);
        }
        if (subs) {
#pragma unroll
            for (int v = 0; v < VPL; ++v) {
                const float qe = q[v] + qf[v];
                float pe = pu[v] + dv * p2[v], se = su[v];
                if (per_day) {
                    pe += pd[v];
                    se += sd[v];
                }
                mf += pe * qe;
                ns += se * qe;
            }
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) {
                float pe = (pu[v] + su[v]) + dv * p2[v];
                if (per_day) {
                    pe += pd[v];
                    pe += sd[v];
                }
                part += pe * (q[v] + qf[v]);
            }
        }
    }
    if (subs) {
        mf = warp_sum(mf);
        ns = warp_sum(ns);
        subs[0] = s.gbias + ubu + ibi + ibf + but + al * dv + bu_day + bit + bi_t * (cu_t - 1.0f) + ycb;
        subs[1] = mf;
        subs[2] = ns;
    } else {
        dot = warp_sum(part);
        bias_part = s.gbias + bu_t + bi_t * cu_t;
    }
}

// u (and i) index the model's user (and item) tables; negative values arrive
// here as large unsigned ones.
__device__ __forceinline__ bool row_in_range(const DeviceState& s, uint32_t u, uint32_t i) {
    return u < s.n_users && i < s.n_items;
}

template <int VPL>
__global__ void __launch_bounds__(kThreads) k_predict(DeviceState s, PredParams pp, const int32_t* __restrict__ u,
                                                      const int32_t* __restrict__ it, const int16_t* __restrict__ d,
                                                      const float* __restrict__ offset, uint64_t n,
                                                      float* __restrict__ out, int subscores) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * kWarps;
    for (uint64_t r = blockIdx.x * (uint64_t)kWarps + (threadIdx.x >> 5); r < n; r += warps) {
        float bp = 0.0f, dot = 0.0f, sub[3];
        const uint32_t ur = (uint32_t)u[r], ir = (uint32_t)it[r];
        if (!row_in_range(s, ur, ir)) {
            // an index outside the model's tables: no table is read, the row's
            // outputs are NaN (device entry points cannot raise per row)
            if (lane == 0) {
                if (subscores) out[3 * r] = out[3 * r + 1] = out[3 * r + 2] = __int_as_float(0x7fc00000);
                else out[r] = __int_as_float(0x7fc00000);
            }
            continue;
        }
        predict_row<VPL>(s, pp, ur, ir, d[r], lane, bp, dot, subscores ? sub : nullptr);
        if (lane == 0) {
            if (subscores) {
                out[3 * r] = sub[0];
                out[3 * r + 1] = sub[1];
                out[3 * r + 2] = sub[2];
            } else {
                const float score = finish_score(s, pp, bp, dot);
                out[r] = offset ? score + offset[r] : score;
            }
        }
    }
}

template <int VPL>
__global__ void __launch_bounds__(kThreads) k_sse(DeviceState s, PredParams pp, const int32_t* __restrict__ u,
                                                  const int32_t* __restrict__ it, const int16_t* __restrict__ d,
                                                  const float* __restrict__ target, const int8_t* __restrict__ is_test,
                                                  uint64_t n, double* __restrict__ part_sse,
                                                  double* __restrict__ part_cnt) {
    __shared__ double ssh[kWarps], csh[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t warps = (uint64_t)gridDim.x * kWarps;
    double sse = 0.0, cnt = 0.0;
    for (uint64_t r = blockIdx.x * (uint64_t)kWarps + warp; r < n; r += warps) {
        if (is_test && is_test[r] != 0) continue;
        if (!row_in_range(s, (uint32_t)u[r], (uint32_t)it[r])) continue;  // the host checked the rows
        float bp = 0.0f, dot = 0.0f;
        predict_row<VPL>(s, pp, (uint32_t)u[r], (uint32_t)it[r], d[r], lane, bp, dot, nullptr);
        const float e = finish_score(s, pp, bp, dot) - target[r];
        const double ed = (double)e;
        sse += ed * ed;
        cnt += 1.0;
    }
    if (lane == 0) {
        ssh[warp] = sse;
        csh[warp] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            a += ssh[w];
            c += csh[w];
        }
        part_sse[blockIdx.x] = a;
        part_cnt[blockIdx.x] = c;
    }
}

__global__ void k_sse_final(const double* __restrict__ ps, const double* __restrict__ pc, unsigned nb,
                            double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (unsigned b = 0; b < nb; ++b) {
            a += ps[b];
            c += pc[b];
        }
        out[0] = a;
        out[1] = c;
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

}  // namespace

void predict_device(const tsvd_model* mc, const int32_t* u, const int32_t* i, const int16_t* day, const float* offset,
                    uint64_t n, float* out, int subscores) {
    tsvd_model* m = const_cast<tsvd_model*>(mc);
    if (n == 0) return;
    ProfScope ps(m, subscores ? "predict_subscores" : "predict");
    PredParams pp{m->cfg.beta, m->cfg.low_memory, m->cfg.has_ordinal_head};
    const int vpl = (int)std::min<uint32_t>(m->d.Fs / 32, 8);
    unsigned grid = (unsigned)std::min<uint64_t>((n + kWarps - 1) / kWarps, 148ull * 16);
    TSVD_DISPATCH(vpl, (k_predict<V><<<grid, kThreads, 0, m->stream>>>(m->d, pp, u, i, day, offset, n, out, subscores)));
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

void sse_device(const tsvd_model* mc, const int32_t* u, const int32_t* i, const int16_t* day, const float* target,
                const int8_t* is_test, uint64_t n, double* out_sse, double* out_cnt) {
    tsvd_model* m = const_cast<tsvd_model*>(mc);
    ProfScope ps(m, "sse");
    PredParams pp{m->cfg.beta, m->cfg.low_memory, m->cfg.has_ordinal_head};
    const int vpl = (int)std::min<uint32_t>(m->d.Fs / 32, 8);
    // the block partials in the model's scratch (allocated on the first call)
    const size_t need = (2 * kSseBlocks + 2) * sizeof(double);
    if (m->m_scratch.bytes < need) m->m_scratch.alloc(need);
    double* psse = m->m_scratch.as<double>();
    double* pcnt = psse + kSseBlocks;
    double* fin = pcnt + kSseBlocks;
    TSVD_DISPATCH(vpl, (k_sse<V><<<kSseBlocks, kThreads, 0, m->stream>>>(m->d, pp, u, i, day, target, is_test, n, psse,
                                                                         pcnt)));
    k_sse_final<<<1, 32, 0, m->stream>>>(psse, pcnt, kSseBlocks, fin);
    TSVD_CUDA(cudaGetLastError());
    m->launches += 2;
    double h[2];
    TSVD_CUDA(cudaMemcpyAsync(h, fin, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
    TSVD_CUDA(cudaStreamSynchronize(m->stream));
    *out_sse = h[0];
    *out_cnt = h[1];
}

}  // namespace tsvd

// ===========================================================================
// Allocation-free RMSE over device-resident rows.
//
// Some callers cannot allocate device memory at the time they need an
// evaluation: a serving process whose memory is reserved up front by its
// owner, code that runs under a caching allocator it must not bypass, or a
// caller that sets all memory aside before a long job and forbids
// cudaMalloc/cudaFree afterwards (both can also synchronise the device, which
// a latency-sensitive caller avoids). tsvd_calc_rmse_device_noalloc serves
// them: the caller passes device inputs and a device output, and the
// reduction's scratch (per-tile partial sums) lives in the file-scope array
// below, which every GPU that loads this library holds until the process
// exits (kNoAllocScratchBytes = 512 KiB).
// ===========================================================================
namespace tsvd {
namespace {

constexpr uint32_t kNoAllocTileRows = 4096;   // rows per fixed tile (one block)
constexpr uint32_t kNoAllocMaxTiles = 32768;  // => at most 134,217,728 rows per call
constexpr uint64_t kNoAllocMaxRows = (uint64_t)kNoAllocTileRows * kNoAllocMaxTiles;

}  // namespace
}  // namespace tsvd

// [2 * tile] = sum of squared errors of tile, [2 * tile + 1] = its row count.
static __device__ __align__(256) double g_noalloc_scratch[2 * tsvd::kNoAllocMaxTiles];

namespace tsvd {
namespace {

constexpr size_t kNoAllocScratchBytes = sizeof(double) * 2 * kNoAllocMaxTiles;
static_assert(kNoAllocScratchBytes == 512 * 1024, "documented scratch size");

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[256] = {};  // device address of the scratch, per device ordinal

// The scratch's device address on the current device. The array's name in host
// code is only a host-side stand-in, so the address is looked up once per
// device, with that device current, and cached.
double* noalloc_scratch(int dev) {
    if (dev < 0 || dev >= 256) throw Error(TSVD_ERR_INVALID, "device ordinal out of range for the no-alloc scratch");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw Error(TSVD_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = (double*)p;
    }
    return g_noalloc_ptr[dev];
}

// One block per fixed tile of kNoAllocTileRows rows; warps take rows
// w, w + 8, ...; the block's sums are combined in warp order. Every tile writes
// both of its slots, so no slot needs clearing between calls.
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_sse_tiles(DeviceState s, PredParams pp, const int32_t* __restrict__ u,
                                                        const int32_t* __restrict__ it, const int16_t* __restrict__ d,
                                                        const float* __restrict__ target,
                                                        const int8_t* __restrict__ is_test, uint64_t n,
                                                        double* __restrict__ part) {
    __shared__ double ssh[kWarps], csh[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t lo = (uint64_t)blockIdx.x * kNoAllocTileRows;
    const uint64_t hi = lo + kNoAllocTileRows < n ? lo + kNoAllocTileRows : n;
    __shared__ double bsh[kWarps];
    double sse = 0.0, cnt = 0.0, bad = 0.0;
    for (uint64_t r = lo + warp; r < hi; r += kWarps) {
        if (is_test && is_test[r] != 0) continue;
        if (!row_in_range(s, (uint32_t)u[r], (uint32_t)it[r])) {
            bad += 1.0;  // never read: counted and reported instead
            continue;
        }
        float bp = 0.0f, dot = 0.0f;
        predict_row<VPL>(s, pp, (uint32_t)u[r], (uint32_t)it[r], d[r], lane, bp, dot, nullptr);
        const double ed = (double)(finish_score(s, pp, bp, dot) - target[r]);
        sse += ed * ed;
        cnt += 1.0;
    }
    if (lane == 0) {
        ssh[warp] = sse;
        csh[warp] = cnt;
        bsh[warp] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0, b = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            a += ssh[w];
            c += csh[w];
            b += bsh[w];
        }
        // a tile with out-of-range rows stores minus their number as its count
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b > 0.0 ? -b : c;
    }
}

// Sums the tiles in order; out = {rmse, sse, count}, or {NaN, NaN, -rows out
// of range} when any row's user or item index was out of range.
__global__ void k_sse_tiles_final(const double* __restrict__ part, uint32_t tiles, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0, c = 0.0, b = 0.0;
        for (uint32_t t = 0; t < tiles; ++t) {
            const double ct = part[2 * t + 1];
            if (ct < 0.0) b -= ct;
            else {
                a += part[2 * t];
                c += ct;
            }
        }
        if (b > 0.0) {
            out[0] = out[1] = __longlong_as_double(0x7ff8000000000000ll);
            out[2] = -b;
        } else {
            out[0] = sqrt(a / c);
            out[1] = a;
            out[2] = c;
        }
    }
}

}  // namespace
}  // namespace tsvd

extern "C" int tsvd_calc_rmse_device_noalloc(const tsvd_model* m, const int32_t* d_u, const int32_t* d_i,
                                             const int16_t* d_day, const float* d_target, const int8_t* d_is_test,
                                             uint64_t n, double* d_out) {
    using namespace tsvd;
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (!d_u || !d_i || !d_day || !d_target || !d_out) throw Error(TSVD_ERR_INVALID, "null device pointer");
        if (n == 0) throw Error(TSVD_ERR_INVALID, "no rows");
        if (n > kNoAllocMaxRows)
            throw Error(TSVD_ERR_INVALID, "tsvd_calc_rmse_device_noalloc: " + std::to_string(n) +
                                              " rows exceed the maximum of " + std::to_string(kNoAllocMaxRows) +
                                              " (its fixed scratch holds " + std::to_string(kNoAllocMaxTiles) +
                                              " tiles of " + std::to_string(kNoAllocTileRows) + " rows)");
        use_device(m);
        double* part = noalloc_scratch(m->device);
        const uint32_t tiles = (uint32_t)((n + kNoAllocTileRows - 1) / kNoAllocTileRows);
        PredParams pp{m->cfg.beta, m->cfg.low_memory, m->cfg.has_ordinal_head};
        const int vpl = (int)std::min<uint32_t>(m->d.Fs / 32, 8);
        TSVD_DISPATCH(vpl, (k_sse_tiles<V><<<tiles, kThreads, 0, m->stream>>>(m->d, pp, d_u, d_i, d_day, d_target,
                                                                              d_is_test, n, part)));
        k_sse_tiles_final<<<1, 32, 0, m->stream>>>(part, tiles, d_out);
        TSVD_CUDA(cudaGetLastError());
        const_cast<tsvd_model*>(m)->launches += 2;
    });
}
