// Deterministic stratified schedule: the reference's own parallel epoch,
// Tsvdx4pModel::fit_epoch (src/tsvdx4p.rs:390-805):
//   user stratum  (fit_epoch_user, :390-639)  users in parallel, item tables
//                 frozen, per-user NSVD1 gradients kept for the delta sums;
//   delta apply   (apply_nsvd_deltas, :341-385) per-item sums over the item's
//                 users in by-item order, split into fixed chunks;
//   ycache rebuild (:267-300);
//   item stratum  (fit_epoch_item, :644-762)  items in parallel, user tables
//                 frozen.
// No two work units touch the same parameter and every sum has a fixed
// order, so a run is bitwise reproducible.
//
// Precision form: with BF16 read copies, the frozen tables a stratum only
// reads are gathered as BF16 (item rows q_i, q^f_{i,0} and y_j; optionally
// the user rows p_u, p2_u, ycache_u of the item stratum) and widened to FP32
// for accumulation; masters stay FP32 and are the only tables written.
#include <mutex>
#include <string>
#include <vector>

#include "rand_stream.hpp"
#include "tsvd_epoch.cuh"

namespace tsvd {
namespace {

// ---------------------------------------------------------------------------
// FP32 -> BF16 read copies (round to nearest even). `src_stride` lets the
// frequency-bin-0 rows of ifeat_freq ([I*NF, Fs]) be copied as an [I, Fs] table.
// ---------------------------------------------------------------------------
__global__ void k_to_bf16(const float* __restrict__ src, uint64_t rows, uint32_t Fs, uint64_t src_stride,
                          __nv_bfloat16* __restrict__ dst) {
    const uint64_t n = rows * Fs;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = e / Fs, c = e - r * Fs;
        dst[e] = __float2bfloat16_rn(src[r * src_stride + c]);
    }
}

template <int VPL, bool BF>
__device__ __forceinline__ void item_rows(const DeviceState& s, const Bf16Copies& bf, uint32_t i, int lane,
                                          float (&q)[VPL], float (&qf)[VPL]) {
    if constexpr (BF) {
        row_load_bf16<VPL>(bf.ifeat + (size_t)i * s.Fs, lane, q);
        row_load_bf16<VPL>(bf.qf0 + (size_t)i * s.Fs, lane, qf);
    } else {
        Row<VPL>::load_nc(s.ifeat + (size_t)i * s.Fs, lane, q);
        Row<VPL>::load_nc(s.ifeat_freq + (size_t)i * s.NF * s.Fs, lane, qf);
    }
}

// su gather with 8 rows in flight (FP32 or BF16 y rows), in the reference's order.
template <int VPL, bool BF, class ItemOf>
__device__ __forceinline__ void gather_y_ro(const DeviceState& s, const Bf16Copies& bf, uint64_t n, ItemOf item_of,
                                            int lane, float (&su)[VPL], float& sub) {
    constexpr int B = 8;
    for (uint64_t base = 0; base < n; base += 32) {
        const uint32_t cnt = (uint32_t)(n - base < 32 ? n - base : 32);
        const uint32_t mine = lane < (int)cnt ? item_of(base + lane) : 0u;
        for (uint32_t j = 0; j < cnt; j += B) {
            float y[B][VPL], yb[B];
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const uint32_t it = __shfl_sync(kFull, mine, j + q < cnt ? j + q : cnt - 1);
                if constexpr (BF) row_load_bf16<VPL>(bf.yfeat + (size_t)it * s.Fs, lane, y[q]);
                else Row<VPL>::load_nc(s.yfeat + (size_t)it * s.Fs, lane, y[q]);
                yb[q] = __ldg(s.ybias + it);
            }
#pragma unroll
            for (int q = 0; q < B; ++q) {
                if (j + q < cnt) {
#pragma unroll
                    for (int v = 0; v < VPL; ++v) su[v] += y[q][v];
                    sub += yb[q];
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// User stratum. Item tables are read-only here; the item rows of rating j+1
// are requested before rating j is used.
// ---------------------------------------------------------------------------
template <int VPL, bool BF>
__global__ void __launch_bounds__(kThreads) k_user_strat(DeviceState s, EpochParams p, Bf16Copies bf,
                                                         const uint32_t* __restrict__ order, uint32_t n_work) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&s.counters[0], 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= n_work) break;
        const uint32_t u = order[k];
        const uint64_t start = s.user_off[u], end = s.user_off[u + 1];
        if (start == end) continue;
        const uint64_t ps = s.pr_off[u], pe = s.pr_off[u + 1];
        const uint64_t total = (end - start) + (p.full_su ? (pe - ps) : 0);
        const float norm = sqrtf((float)total);

        // su (src/tsvdx4p.rs:466-491): equals ycache[u] bit for bit when full_su
        // holds and ycache was rebuilt from the current y.
        float su[VPL], sub;
        if (p.use_ycache) {
            Row<VPL>::load_cg(s.ycache + (size_t)u * Fs, lane, su);
            sub = __ldcg(s.ycache_bias + u);
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = 0.0f;
            sub = 0.0f;
            const Rec* rr = s.rec + start;
            gather_y_ro<VPL, BF>(s, bf, end - start, [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su,
                                 sub);
            if (p.full_su) {
                const uint32_t* pp = s.pr_item + ps;
                gather_y_ro<VPL, BF>(s, bf, pe - ps, [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sub);
            }
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = su[v] / norm;
            sub = sub / norm;
            Row<VPL>::store(s.ycache + (size_t)u * Fs, lane, su);
            if (lane == 0) s.ycache_bias[u] = sub;
        }

        float pu[VPL], p2[VPL], seq[VPL];
        Row<VPL>::load_cg(s.ufeat + (size_t)u * Fs, lane, pu);
        Row<VPL>::load_cg(s.ufeat2 + (size_t)u * Fs, lane, p2);
#pragma unroll
        for (int v = 0; v < VPL; ++v) seq[v] = 0.0f;
        float ub = __ldcg(s.ubias + u), al = __ldcg(s.alpha_u + u), cuu = __ldcg(s.cu + u);
        float bb0 = lane < (int)T ? __ldcg(s.but_bin + (size_t)u * T + lane) : 0.0f;
        float bb1 = lane + 32 < (int)T ? __ldcg(s.but_bin + (size_t)u * T + 32 + lane) : 0.0f;
        float sum_err = 0.0f;
        const float gb = s.gbias;

        for (uint64_t base = start; base < end; base += 32) {
            const uint32_t cnt = (uint32_t)(end - base < 32 ? end - base : 32);
            Rec mine{};
            if (lane < (int)cnt) mine = load_rec(s.rec + base + lane);
            float qn[VPL], qfn[VPL];
            item_rows<VPL, BF>(s, bf, rec_id(__shfl_sync(kFull, mine.key, 0)), lane, qn, qfn);
            for (uint32_t j = 0; j < cnt; ++j) {
                const Rec r = shfl_rec(mine, j);
                const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
                float q[VPL], qf[VPL];
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    q[v] = qn[v];
                    qf[v] = qfn[v];
                }
                if (j + 1 < cnt) item_rows<VPL, BF>(s, bf, rec_id(__shfl_sync(kFull, mine.key, j + 1)), lane, qn, qfn);
                // low_memory: training uses frequency bin 0 (src/tsvdx4p.rs:504-531)
                const float ib = __ldg(s.ibias + i);
                const float bit = __ldg(s.bit_bin + (size_t)i * T + tb);
                const float ibf = __ldg(s.ibias_freq + (size_t)i * NF);
                const bool hud = r.ud < s.n_ud;
                float bud = 0.0f;
                if (lane == 0 && hud) bud = s.ubias_day[r.ud];
                bud = __shfl_sync(kFull, bud, 0);
                const float ct = hud ? __ldg(s.cut + r.ud) : 0.0f;
                const float but = __shfl_sync(kFull, tb < 32 ? bb0 : bb1, tb & 31);
                const float dv = r.dev;
                const float bu_t = ub + but + al * dv + bud + sub;
                const float bi_t = ib + bit + ibf;
                const float cu_t = cuu + ct;
                float part = 0.0f;
#pragma unroll
                for (int v = 0; v < VPL; ++v) part += (q[v] + qf[v]) * ((pu[v] + su[v]) + dv * p2[v]);
                const float dot = warp_sum(part);
                const float err = (gb + bu_t + bi_t * cu_t + dot) - r.res;
                ub -= p.lr_ub * err;
                {
                    const float nb = but - p.lr_tu * err;
                    if (lane == (int)(tb & 31)) {
                        if (tb < 32) bb0 = nb;
                        else bb1 = nb;
                    }
                }
                al -= p.lr_ta * err * dv;
                if (lane == 0 && hud) s.ubias_day[r.ud] = bud - p.lr_ubd * err;
                cuu -= p.lr_cu * (err * bi_t + p.reg_cu * (cuu - 1.0f));
                sum_err += err;
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    const float qe = q[v] + qf[v];
                    const float pk = pu[v], p2k = p2[v];
                    seq[v] += err * qe;
                    pu[v] = pk - p.lr_u * (err * qe + p.reg_u * pk);
                    p2[v] = p2k - p.lr_u2 * (err * qe * dv + p.reg_u2 * p2k);
                }
            }
        }
        Row<VPL>::store(s.ufeat + (size_t)u * Fs, lane, pu);
        Row<VPL>::store(s.ufeat2 + (size_t)u * Fs, lane, p2);
        if (lane == 0) {
            s.ubias[u] = ub;
            s.alpha_u[u] = al;
            s.cu[u] = cuu;
        }
        if (lane < (int)T) s.but_bin[(size_t)u * T + lane] = bb0;
        if (lane + 32 < (int)T) s.but_bin[(size_t)u * T + 32 + lane] = bb1;
        float g[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) g[v] = seq[v] / norm;
        Row<VPL>::store(s.g_user + (size_t)u * Fs, lane, g);
        if (lane == 0) s.e_user[u] = sum_err / norm;
    }
}

// ---------------------------------------------------------------------------
// NSVD1 delta sums per item in two fixed-order levels: fixed chunks of
// kChunkUsers consecutive by-item entries are summed by one warp each
// (k_y_partial), then each item adds its chunk partials in chunk order and
// applies the update (k_y_combine).
// ---------------------------------------------------------------------------
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_y_partial(DeviceState s) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs;
    constexpr int B = 8;  // rows in flight per warp
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&s.counters[1], 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= s.n_chunks) break;
        const uint64_t a = s.chunk_lo[c];
        uint64_t b = s.chunk_lo[c + 1];
        if (b - a > kChunkUsers) b = a + kChunkUsers;
        float acc[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) acc[v] = 0.0f;
        float eacc = 0.0f;
        for (uint64_t base = a; base < b; base += 32) {
            const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
            const uint32_t mine = lane < (int)cnt ? rec_id(__ldg(&s.irec[base + lane].key)) : 0u;
            for (uint32_t j = 0; j < cnt; j += B) {
                float g[B][VPL], e[B];
#pragma unroll
                for (int q = 0; q < B; ++q) {
                    const uint32_t u = __shfl_sync(kFull, mine, j + q < cnt ? j + q : cnt - 1);
                    Row<VPL>::load_nc(s.g_user + (size_t)u * Fs, lane, g[q]);
                    e[q] = __ldg(s.e_user + u);
                }
#pragma unroll
                for (int q = 0; q < B; ++q) {
                    if (j + q < cnt) {
#pragma unroll
                        for (int v = 0; v < VPL; ++v) acc[v] += g[q][v];
                        eacc += e[q];
                    }
                }
            }
        }
        Row<VPL>::store(s.chunk_part + (size_t)c * Fs, lane, acc);
        if (lane == 0) s.chunk_epart[c] = eacc;
    }
}

template <int VPL>
__global__ void __launch_bounds__(kThreads) k_y_combine(DeviceState s, EpochParams p) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs;
    const uint32_t warps = gridDim.x * kWarps;
    for (uint32_t i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < s.n_items; i += warps) {
        const uint32_t c0 = s.item_chunk0[i], c1 = s.item_chunk0[i + 1];
        if (c0 == c1) continue;
        float acc[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) acc[v] = 0.0f;
        float eacc = 0.0f;
        for (uint32_t c = c0; c < c1; ++c) {
            float g[VPL];
            Row<VPL>::load_cg(s.chunk_part + (size_t)c * Fs, lane, g);
#pragma unroll
            for (int v = 0; v < VPL; ++v) acc[v] += g[v];
            eacc += __ldcg(s.chunk_epart + c);
        }
        const float nc = (float)(s.item_off[i + 1] - s.item_off[i]);
        const float scale = p.nsvd_norm_exp == 0.0f ? 1.0f : powf(nc, p.nsvd_norm_exp);
        float y[VPL];
        Row<VPL>::load_cg(s.yfeat + (size_t)i * Fs, lane, y);
#pragma unroll
        for (int v = 0; v < VPL; ++v) y[v] = y[v] - p.lr_y * (acc[v] / scale + p.reg_y * y[v]);
        Row<VPL>::store(s.yfeat + (size_t)i * Fs, lane, y);
        if (lane == 0) s.ybias[i] = s.ybias[i] - p.lr_yb * (eacc / scale);
    }
}

// ---------------------------------------------------------------------------
// Item stratum. An item's ratings form a serial chain (every update feeds the
// next dot product), and the most-rated items carry ~0.5% of all ratings
// each, so the chain of the hottest item bounds the pass. Items with >= kHeavy
// ratings get a whole CTA, warp-specialised: warps 1..7 gather the user rows of
// the next round of kRound ratings and fold them into
// pe = (p_u + ycache_u) + dev * p2_u plus the rating's bias scalars in shared
// memory (double-buffered rounds, one __syncthreads per round), while warp 0
// runs the chain from shared memory only. Lighter items take one warp each,
// with the next rating's rows prefetched into registers.
// ---------------------------------------------------------------------------
constexpr uint32_t kHeavy = 1024;
constexpr int kRound = 32;  // ratings per buffered round
constexpr uint32_t kGramStride = kRound + 1;  // padded rows of the per-round Gram matrix

// x = hi + lo with hi, lo in TF32 (round to nearest, ties away from zero).
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    const float rest = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(rest));
}

// d (16x8, FP32) += a (16x8, TF32, row-major) . b (8x8, TF32, column-major)
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

struct ItemState {
    float ib, bt0, bt1, bf0, bf1;
};

__device__ __forceinline__ ItemState load_item_state(const DeviceState& s, uint32_t i, int lane) {
    const uint32_t T = s.T, NF = s.NF;
    ItemState st;
    st.ib = s.ibias[i];
    st.bt0 = lane < (int)T ? s.bit_bin[(size_t)i * T + lane] : 0.0f;
    st.bt1 = lane + 32 < (int)T ? s.bit_bin[(size_t)i * T + 32 + lane] : 0.0f;
    st.bf0 = lane < (int)NF ? s.ibias_freq[(size_t)i * NF + lane] : 0.0f;
    st.bf1 = lane + 32 < (int)NF ? s.ibias_freq[(size_t)i * NF + 32 + lane] : 0.0f;
    return st;
}

__device__ __forceinline__ void store_item_state(const DeviceState& s, uint32_t i, int lane, const ItemState& st) {
    const uint32_t T = s.T, NF = s.NF;
    if (lane == 0) s.ibias[i] = st.ib;
    if (lane < (int)T) s.bit_bin[(size_t)i * T + lane] = st.bt0;
    if (lane + 32 < (int)T) s.bit_bin[(size_t)i * T + 32 + lane] = st.bt1;
    if (lane < (int)NF) s.ibias_freq[(size_t)i * NF + lane] = st.bf0;
    if (lane + 32 < (int)NF) s.ibias_freq[(size_t)i * NF + 32 + lane] = st.bf1;
}

// User-side scalars of one by-item rating: bu_t and cu_t (src/tsvdx4p.rs:690-708).
__device__ __forceinline__ void user_scalars(const DeviceState& s, const Rec& r, float& bu_t, float& cu_t) {
    const uint32_t u = rec_id(r.key), tb = rec_tbin(r.key);
    const bool hud = r.ud < s.n_ud;
    bu_t = __ldg(s.ubias + u) + __ldg(s.but_bin + (size_t)u * s.T + tb) + __ldg(s.alpha_u + u) * r.dev +
           (hud ? __ldg(s.ubias_day + r.ud) : 0.0f) + __ldg(s.ycache_bias + u);
    cu_t = __ldg(s.cu + u) + (hud ? __ldg(s.cut + r.ud) : 0.0f);
}

template <int VPL, bool BF>
__device__ __forceinline__ void user_rows(const DeviceState& s, const Bf16Copies& bf, uint32_t u, int lane,
                                          float (&pu)[VPL], float (&p2)[VPL], float (&yc)[VPL]) {
    if constexpr (BF) {
        row_load_bf16<VPL>(bf.ufeat + (size_t)u * s.Fs, lane, pu);
        row_load_bf16<VPL>(bf.ufeat2 + (size_t)u * s.Fs, lane, p2);
        row_load_bf16<VPL>(bf.ycache + (size_t)u * s.Fs, lane, yc);
    } else {
        Row<VPL>::load_nc(s.ufeat + (size_t)u * s.Fs, lane, pu);
        Row<VPL>::load_nc(s.ufeat2 + (size_t)u * s.Fs, lane, p2);
        Row<VPL>::load_nc(s.ycache + (size_t)u * s.Fs, lane, yc);
    }
}

// One SGD step of the item chain; qf_at(v) is this lane's v-th element of q^f[fb].
template <int VPL, class QF>
__device__ __forceinline__ void item_step(const EpochParams& p, float gb, float (&q)[VPL], QF&& qf_at,
                                          const float (&pe)[VPL], float bu_t, float cu_t, float res, uint32_t tb,
                                          uint32_t fb, int lane, ItemState& st) {
    const float bit = __shfl_sync(kFull, tb < 32 ? st.bt0 : st.bt1, tb & 31);
    const float ibf = __shfl_sync(kFull, fb < 32 ? st.bf0 : st.bf1, fb & 31);
    const float bi_t = st.ib + bit + ibf;
    float qfv[VPL], part = 0.0f;
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
        qfv[v] = qf_at(v);
        part += pe[v] * (q[v] + qfv[v]);
    }
    const float dot = warp_sum(part);
    const float err = (gb + bu_t + bi_t * cu_t + dot) - res;
    const float ec = err * cu_t;
    st.ib -= p.lr_ib * ec;
    const float nb = bit - p.lr_ti * ec;
    if (lane == (int)(tb & 31)) {
        if (tb < 32) st.bt0 = nb;
        else st.bt1 = nb;
    }
    const float nf = ibf - p.lr_ibf * ec;
    if (lane == (int)(fb & 31)) {
        if (fb < 32) st.bf0 = nf;
        else st.bf1 = nf;
    }
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
        const float qi = q[v];
        q[v] = qi - p.lr_i * (err * pe[v] + p.reg_i * qi);
        qfv[v] = qfv[v] - p.lr_iqf * (err * pe[v] + p.reg_iqf * qfv[v]);
    }
#pragma unroll
    for (int v = 0; v < VPL; ++v) qf_at(v) = qfv[v];
}

template <int VPL, bool BF>
__device__ void item_light(const DeviceState& s, const EpochParams& p, const Bf16Copies& bf, uint32_t i, int lane) {
    const uint32_t Fs = s.Fs, NF = s.NF;
    const uint64_t a = s.item_off[i], b = s.item_off[i + 1];
    if (a == b) return;
    float q[VPL];
    Row<VPL>::load_cg(s.ifeat + (size_t)i * Fs, lane, q);
    ItemState st = load_item_state(s, i, lane);
    float* qf_base = s.ifeat_freq + (size_t)i * NF * Fs;
    const float gb = s.gbias;
    for (uint64_t base = a; base < b; base += 32) {
        const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
        Rec mine{};
        if (lane < (int)cnt) mine = load_rec(s.irec + base + lane);
        float pn[VPL], p2n[VPL], ycn[VPL];
        user_rows<VPL, BF>(s, bf, rec_id(__shfl_sync(kFull, mine.key, 0)), lane, pn, p2n, ycn);
        for (uint32_t j = 0; j < cnt; ++j) {
            const Rec r = shfl_rec(mine, j);
            float pe[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) pe[v] = (pn[v] + ycn[v]) + r.dev * p2n[v];
            if (j + 1 < cnt) user_rows<VPL, BF>(s, bf, rec_id(__shfl_sync(kFull, mine.key, j + 1)), lane, pn, p2n, ycn);
            float bu_t, cu_t;
            user_scalars(s, r, bu_t, cu_t);
            const uint32_t tb = rec_tbin(r.key), fb = rec_fbin(r.key);
            float* qrow = qf_base + (size_t)fb * Fs;
            float qfv[VPL];
            Row<VPL>::load_cg(qrow, lane, qfv);
            item_step<VPL>(p, gb, q, [&](int v) -> float& { return qfv[v]; }, pe, bu_t, cu_t, r.res, tb, fb, lane,
                           st);
            Row<VPL>::store(qrow, lane, qfv);
        }
    }
    Row<VPL>::store(s.ifeat + (size_t)i * Fs, lane, q);
    store_item_state(s, i, lane, st);
}

template <int VPL, bool BF>
__global__ void __launch_bounds__(kThreads, 2) k_item_pass(DeviceState s, EpochParams p, Bf16Copies bf) {
    extern __shared__ float smem[];
    __shared__ uint32_t sh_k;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t Fs = s.Fs, NF = s.NF;
    const uint32_t stride = Fs + 4;       // one staged rating: pe row + {bu_t, cu_t, res, key}
    const uint32_t qs = Fs + 4;           // padded q^f row stride (rows of different bins in distinct banks)
    float* qfs = smem;                    // [NF][qs]
    float* qsh = qfs + (size_t)NF * qs;   // [Fs] q row of the current round
    float* buf = qsh + Fs;                // [2][kRound][stride]
    float* gram = buf + 2ull * kRound * stride;  // [2][kRound][kGramStride]
    for (;;) {
        if (threadIdx.x == 0) sh_k = atomicAdd(&s.counters[2], 1u);
        __syncthreads();
        const uint32_t k = sh_k;
        __syncthreads();
        if (k >= s.n_items) return;
        const uint32_t i = s.item_work[k];
        const uint64_t a = s.item_off[i], b = s.item_off[i + 1];
        if (b - a < kHeavy) {
            // Items are ordered heaviest first: from here on every item is light.
            if (warp == 0) item_light<VPL, BF>(s, p, bf, i, lane);
            for (;;) {
                uint32_t k2 = 0;
                if (lane == 0) k2 = atomicAdd(&s.counters[2], 1u);
                k2 = __shfl_sync(kFull, k2, 0);
                if (k2 >= s.n_items) return;
                item_light<VPL, BF>(s, p, bf, s.item_work[k2], lane);
            }
        }
        // ---------------- heavy item: whole CTA ----------------
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            qfs[(e / Fs) * qs + e % Fs] = __ldcg(s.ifeat_freq + (size_t)i * NF * Fs + e);
        const uint64_t n = b - a;
        const uint32_t rounds = (uint32_t)((n + kRound - 1) / kRound);
        float q[VPL];
        ItemState st{};
        if (warp == 0) {
            Row<VPL>::load_cg(s.ifeat + (size_t)i * Fs, lane, q);
            st = load_item_state(s, i, lane);
        }
        auto round_len = [&](uint32_t r) -> uint32_t {
            const uint64_t left = n - (uint64_t)r * kRound;
            return (uint32_t)(left < (uint64_t)kRound ? left : (uint64_t)kRound);
        };
        auto produce = [&](uint32_t r) {
            float* dst = buf + (size_t)(r & 1) * kRound * stride;
            const uint64_t r0 = a + (uint64_t)r * kRound;
            const uint32_t m = round_len(r);
            // the round's records and user-side scalars, one rating per lane
            Rec mine{};
            float bu_l = 0.0f, cu_l = 0.0f;
            if ((uint32_t)lane < m) {
                mine = load_rec(s.irec + r0 + lane);
                user_scalars(s, mine, bu_l, cu_l);
            }
            auto put = [&](uint32_t j, const float (&pu)[VPL], const float (&p2)[VPL], const float (&yc)[VPL]) {
                const float dev = __shfl_sync(kFull, mine.dev, j), bu = __shfl_sync(kFull, bu_l, j);
                const float cu = __shfl_sync(kFull, cu_l, j), res = __shfl_sync(kFull, mine.res, j);
                const uint32_t key = __shfl_sync(kFull, mine.key, j);
                float* row = dst + (size_t)j * stride;
#pragma unroll
                for (int v = 0; v < VPL; ++v) row[Row<VPL>::elem(lane, v)] = (pu[v] + yc[v]) + dev * p2[v];
                if (lane == 0) {
                    row[Fs] = bu;
                    row[Fs + 1] = cu;
                    row[Fs + 2] = res;
                    row[Fs + 3] = __uint_as_float(key);
                }
            };
            // user rows of two ratings in flight per warp
            for (uint32_t j0 = warp - 1; j0 < m; j0 += 2 * (kWarps - 1)) {
                const uint32_t j1 = j0 + (kWarps - 1);
                const bool two = j1 < m;
                const uint32_t u0 = rec_id(__shfl_sync(kFull, mine.key, j0));
                const uint32_t u1 = rec_id(__shfl_sync(kFull, mine.key, two ? j1 : j0));
                float pa[VPL], p2a[VPL], yca[VPL], pb[VPL], p2b[VPL], ycb[VPL];
                user_rows<VPL, BF>(s, bf, u0, lane, pa, p2a, yca);
                if (two) user_rows<VPL, BF>(s, bf, u1, lane, pb, p2b, ycb);
                put(j0, pa, p2a, yca);
                if (two) put(j1, pb, p2b, ycb);
            }
            // rows m..31 of a partial round are zero (finite values for the
            // consumer's unconditional loops)
            for (uint32_t j = m + warp - 1; j < (uint32_t)kRound; j += kWarps - 1) {
                float* row = dst + (size_t)j * stride;
                for (uint32_t e = lane; e < stride; e += 32) row[e] = 0.0f;
            }
            // all rows of the round are in place before the Gram products
            asm volatile("bar.sync 1, %0;" ::"r"((kWarps - 1) * 32) : "memory");
            // G = PE PE^T for the round's ratings, on the tensor cores: TF32
            // operands split into high and low parts, three products per
            // tile (error near FP32's). Producer warp w takes tile w - 1 of
            // the six 16x8 tiles that hold the pairs k < j.
            const int tile = warp - 1;
            if (tile < 6) {
                float* gm = gram + (size_t)(r & 1) * kRound * kGramStride;
                const int mt = tile < 4 ? 0 : 1, nt = tile < 4 ? tile : tile - 2;
                const int gid = lane >> 2, tig = lane & 3;
                const float* A0 = dst + (size_t)(mt * 16 + gid) * stride;
                const float* A1 = A0 + 8 * (size_t)stride;
                const float* B0 = dst + (size_t)(nt * 8 + gid) * stride;
                // independent accumulators: the three split products and
                // even/odd k-steps run as separate MMA chains
                float d[6][4] = {};
#pragma unroll 2
                for (uint32_t k0 = 0; k0 < Fs; k0 += 16) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t kk = k0 + 8 * h;
                        uint32_t ah[4], al[4], bh[2], bl[2];
                        split_tf32(A0[kk + tig], ah[0], al[0]);
                        split_tf32(A1[kk + tig], ah[1], al[1]);
                        split_tf32(A0[kk + tig + 4], ah[2], al[2]);
                        split_tf32(A1[kk + tig + 4], ah[3], al[3]);
                        split_tf32(B0[kk + tig], bh[0], bl[0]);
                        split_tf32(B0[kk + tig + 4], bh[1], bl[1]);
                        mma_tf32(d[3 * h], al, bh);
                        mma_tf32(d[3 * h + 1], ah, bl);
                        mma_tf32(d[3 * h + 2], ah, bh);
                    }
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) d[0][e] = ((d[0][e] + d[1][e]) + (d[3][e] + d[4][e])) + (d[2][e] + d[5][e]);
                float* g0 = gm + (size_t)(mt * 16 + gid) * kGramStride + nt * 8 + 2 * tig;
                g0[0] = d[0][0];
                g0[1] = d[0][1];
                g0[8 * kGramStride] = d[0][2];
                g0[8 * kGramStride + 1] = d[0][3];
            }
        };
        if (warp > 0) produce(0);
        __syncthreads();
        const float gb = s.gbias;
        // update factors: x - lr (g + reg x) = a x - lr g
        const float a_i = 1.0f - p.lr_i * p.reg_i, a_f = 1.0f - p.lr_iqf * p.reg_iqf;
        for (uint32_t r = 0; r < rounds; ++r) {
            if (warp > 0) {
                if (r + 1 < rounds) produce(r + 1);
            } else {
                // Lookahead over the round's m ratings (all of one item): with
                // q_k, qf_k the item rows before rating k, and pe_k fixed in
                // the item stratum,
                //   q_k . pe_k = a_i^k (q_0 . pe_k) - lr_i sum_{j<k} a_i^(k-1-j) err_j G_jk
                // and likewise for the q^f row of pe_k's frequency bin over the
                // earlier ratings of the same bin. The dots with q_0 are taken
                // once per round; the serial chain is then scalar per rating,
                // and the round's updates are applied in closed form,
                //   q_m = a_i^m q_0 - lr_i sum_k a_i^(m-1-k) err_k pe_k.
                // Rows m..31 of a partial round are zero.
                const float* src = buf + (size_t)(r & 1) * kRound * stride;
                const float* gm = gram + (size_t)(r & 1) * kRound * kGramStride;
                const uint32_t m = round_len(r);
                const float* myrow = src + (size_t)lane * stride;
                const float bu_t = myrow[Fs], cu_t = myrow[Fs + 1], res = myrow[Fs + 2];
                const uint32_t key = __float_as_uint(myrow[Fs + 3]);
                const uint32_t tb = rec_tbin(key), fb = rec_fbin(key);
                // this lane's dots with q_0 and q^f_0[fb]: the round's q row
                // goes to shared memory, and each lane walks its own pe row
#pragma unroll
                for (int v = 0; v < VPL; ++v) qsh[Row<VPL>::elem(lane, v)] = q[v];
                __syncwarp();
                float sq, sf;
                {
                    const float4* x4 = reinterpret_cast<const float4*>(myrow);
                    const float4* y4 = reinterpret_cast<const float4*>(qsh);
                    const float4* z4 = reinterpret_cast<const float4*>(qfs + (size_t)fb * qs);
                    float s0 = 0.0f, s1 = 0.0f, e0 = 0.0f, e1 = 0.0f;
#pragma unroll 4
                    for (uint32_t k4 = 0; k4 < Fs / 4; ++k4) {
                        const float4 x = x4[k4], y = y4[k4], z = z4[k4];
                        s0 = fmaf(x.x, y.x, s0);
                        s1 = fmaf(x.y, y.y, s1);
                        s0 = fmaf(x.z, y.z, s0);
                        s1 = fmaf(x.w, y.w, s1);
                        e0 = fmaf(x.x, z.x, e0);
                        e1 = fmaf(x.y, z.y, e1);
                        e0 = fmaf(x.z, z.z, e0);
                        e1 = fmaf(x.w, z.w, e1);
                    }
                    sq = s0 + s1;  // q_0 . pe_lane
                    sf = e0 + e1;  // qf_0[fb] . pe_lane
                }
                // The round's errors solve a unit lower-triangular system
                // err = C - M err: C_j holds everything known at the round's
                // start, M_ji (i < j) the effect of err_i on rating j through
                // q, q^f of the same bin and the item biases. Forward
                // substitution then costs one broadcast and one FMA per rating.
                const bool valid = lane < (int)m;
                float Mrow[kRound];
                float pw_d = 1.0f, pwf_d = 1.0f;  // a_i^(j-1-i), a_f^(same-bin ratings between i and j)
#pragma unroll
                for (int i = kRound - 1; i >= 0; --i) {
                    const float gij = gm[i * kGramStride + lane];
                    const float cui = __shfl_sync(kFull, cu_t, i);
                    const uint32_t ti = __shfl_sync(kFull, tb, i), fi = __shfl_sync(kFull, fb, i);
                    const bool before = i < lane, same_f = fi == fb, same_t = ti == tb;
                    const float bias_lr = p.lr_ib + (same_t ? p.lr_ti : 0.0f) + (same_f ? p.lr_ibf : 0.0f);
                    const float v = cu_t * cui * bias_lr + p.lr_i * pw_d * gij + (same_f ? p.lr_iqf * pwf_d * gij : 0.0f);
                    Mrow[i] = before ? v : 0.0f;
                    if (before) {
                        pw_d *= a_i;
                        if (same_f) pwf_d *= a_f;
                    }
                }
                // pw_d = a_i^j, pwf_d = a_f^(earlier ratings of the same bin)
                const float bi0 = st.ib + __shfl_sync(kFull, tb < 32 ? st.bt0 : st.bt1, tb & 31) +
                                  __shfl_sync(kFull, fb < 32 ? st.bf0 : st.bf1, fb & 31);
                float x = ((gb + bu_t + bi0 * cu_t) + (pw_d * sq + pwf_d * sf)) - res;
                x = valid ? x : 0.0f;
#pragma unroll
                for (int i = 0; i < kRound; ++i) x = fmaf(-Mrow[i], __shfl_sync(kFull, x, i), x);
                const float my_err = x, my_ec = x * cu_t;
                // weights of the closed-form updates: a_i^(m-1-j), a_f^(later ratings of the same bin), a_i^m
                float pw = 1.0f, pwf = 1.0f, am = 1.0f;
#pragma unroll
                for (int i = 0; i < kRound; ++i) {
                    const uint32_t fi = __shfl_sync(kFull, fb, i);
                    const bool inr = i < (int)m, after = inr && i > lane;
                    am = inr ? am * a_i : am;
                    pw = after ? pw * a_i : pw;
                    pwf = (after && fi == fb) ? pwf * a_f : pwf;
                }
                const float wq = valid ? p.lr_i * pw * my_err : 0.0f;
                const float wf = valid ? p.lr_iqf * pwf * my_err : 0.0f;
                const float wb = valid ? my_ec : 0.0f;
                // biases
                st.ib -= p.lr_ib * warp_sum(wb);
                {
                    float dt0 = 0.0f, dt1 = 0.0f, df0 = 0.0f, df1 = 0.0f;
#pragma unroll 4
                    for (int k = 0; k < kRound; ++k) {
                        const float e = __shfl_sync(kFull, wb, k);
                        const uint32_t tbk = __shfl_sync(kFull, tb, k), fbk = __shfl_sync(kFull, fb, k);
                        dt0 += lane == (int)tbk ? e : 0.0f;
                        dt1 += lane + 32 == (int)tbk ? e : 0.0f;
                        df0 += lane == (int)fbk ? e : 0.0f;
                        df1 += lane + 32 == (int)fbk ? e : 0.0f;
                    }
                    st.bt0 -= p.lr_ti * dt0;
                    st.bt1 -= p.lr_ti * dt1;
                    st.bf0 -= p.lr_ibf * df0;
                    st.bf1 -= p.lr_ibf * df1;
                }
                // q
#pragma unroll
                for (int v = 0; v < VPL; ++v) q[v] *= am;
#pragma unroll 4
                for (int k = 0; k < kRound; ++k) {
                    const float w = __shfl_sync(kFull, wq, k);
                    float pk[VPL];
                    row_from_smem<VPL>(src + (size_t)k * stride, lane, pk);
#pragma unroll
                    for (int v = 0; v < VPL; ++v) q[v] = fmaf(-w, pk[v], q[v]);
                }
                // q^f rows: the first rating of a bin also applies the bin's decay
                const unsigned same = __match_any_sync(kFull, valid ? fb : 64u + (uint32_t)lane);
                float dec = 1.0f;
                if (valid && __ffs(same) - 1 == lane)
                    for (int z = __popc(same); z > 0; --z) dec *= a_f;
#pragma unroll 2
                for (int k = 0; k < kRound; ++k) {
                    const float w = __shfl_sync(kFull, wf, k), dk = __shfl_sync(kFull, dec, k);
                    const uint32_t f = __shfl_sync(kFull, fb, k);
                    float* qrow = qfs + (size_t)f * qs;
                    float row[VPL], pk[VPL];
                    row_from_smem<VPL>(qrow, lane, row);
                    row_from_smem<VPL>(src + (size_t)k * stride, lane, pk);
#pragma unroll
                    for (int v = 0; v < VPL; ++v) row[v] = fmaf(-w, pk[v], dk * row[v]);
#pragma unroll
                    for (int v = 0; v < VPL; ++v) qrow[Row<VPL>::elem(lane, v)] = row[v];
                }
                __syncwarp();
            }
            __syncthreads();
        }
        if (warp == 0) {
            Row<VPL>::store(s.ifeat + (size_t)i * Fs, lane, q);
            store_item_state(s, i, lane, st);
        }
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            __stcg(s.ifeat_freq + (size_t)i * NF * Fs + e, qfs[(e / Fs) * qs + e % Fs]);
        __syncthreads();
    }
}

void to_bf16(tsvd_model* m, const float* src, uint64_t rows, uint64_t src_stride, void* dst) {
    const uint32_t Fs = m->d.Fs;
    const unsigned grid = (unsigned)std::min<uint64_t>((rows * Fs + 255) / 256, 148ull * 32);
    k_to_bf16<<<grid, 256, 0, m->stream>>>(src, rows, Fs, src_stride, (__nv_bfloat16*)dst);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL, bool BF, bool BFU>
void strat_launch(tsvd_model* m, const EpochParams& p, const Bf16Copies& bf) {
    const DeviceState& s = m->d;
    {
        ProfScope ps(m, "user_pass_stratified");
        unsigned g = persistent_grid(k_user_strat<VPL, BF>, 0);
        k_user_strat<VPL, BF><<<g, kThreads, 0, m->stream>>>(s, p, bf, s.user_work, s.n_users);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    {
        ProfScope ps(m, "y_apply");
        unsigned g = persistent_grid(k_y_partial<VPL>, 0);
        k_y_partial<VPL><<<g, kThreads, 0, m->stream>>>(s);
        k_y_combine<VPL><<<ceil_div(s.n_items, kWarps), kThreads, 0, m->stream>>>(s, p);
        TSVD_CUDA(cudaGetLastError());
        m->launches += 2;
    }
    if (BF) to_bf16(m, s.yfeat, s.n_items, s.Fs, m->m_bf_yfeat.p);
    launch_rebuild_ycache(m);
    if (BFU) {
        ProfScope ps(m, "bf16_copies");
        to_bf16(m, s.ufeat, s.n_users, s.Fs, m->m_bf_ufeat.p);
        to_bf16(m, s.ufeat2, s.n_users, s.Fs, m->m_bf_ufeat2.p);
        to_bf16(m, s.ycache, s.n_users, s.Fs, m->m_bf_ycache.p);
    }
    {
        ProfScope ps(m, "item_pass");
        const size_t smem =
            ((size_t)s.NF * (s.Fs + 4) + s.Fs + 2ull * kRound * (s.Fs + 4) + 2ull * kRound * kGramStride) *
            sizeof(float);
        TSVD_CUDA(cudaFuncSetAttribute(k_item_pass<VPL, BFU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        unsigned g = persistent_grid(k_item_pass<VPL, BFU>, smem);
        k_item_pass<VPL, BFU><<<g, kThreads, smem, m->stream>>>(s, p, bf);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
}

// Standard init of a set of users: p_u rows given (host-drawn), the rest as
// TxModel::new leaves it (src/tx.rs:600-648).
__global__ void k_reset_users(DeviceState s, const uint32_t* __restrict__ users, uint32_t n,
                              const float* __restrict__ prow) {
    const uint32_t w = blockIdx.x;
    if (w >= n) return;
    const uint32_t u = users[w];
    for (uint32_t c = threadIdx.x; c < s.Fs; c += blockDim.x) {
        s.ufeat[(size_t)u * s.Fs + c] = prow[(size_t)w * s.Fs + c];
        s.ufeat2[(size_t)u * s.Fs + c] = 0.0f;
    }
    for (uint32_t b = threadIdx.x; b < s.T; b += blockDim.x) s.but_bin[(size_t)u * s.T + b] = 0.0f;
    for (uint64_t d = s.ud_start[u] + threadIdx.x; d < s.ud_start[u + 1]; d += blockDim.x) s.ubias_day[d] = 0.0f;
    if (threadIdx.x == 0) {
        s.ubias[u] = 0.0f;
        s.alpha_u[u] = 0.0f;
        s.cu[u] = 1.0f;
    }
}

template <int VPL>
void foldin_launch(tsvd_model* m, const EpochParams& p, const uint32_t* d_users, uint32_t n) {
    unsigned g = persistent_grid(k_user_strat<VPL, false>, 0);
    k_user_strat<VPL, false><<<g, kThreads, 0, m->stream>>>(m->d, p, Bf16Copies{}, d_users, n);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

}  // namespace

void stratified_epoch(tsvd_model* m, const EpochParams& p) {
    const DeviceState& s = m->d;
    const int prec = m->opts.precision;
    Bf16Copies bf{};
    if (prec >= TSVD_PREC_BF16_READ) {
        ProfScope ps(m, "bf16_copies");
        to_bf16(m, s.ifeat, s.n_items, s.Fs, m->m_bf_ifeat.p);
        to_bf16(m, s.ifeat_freq, s.n_items, (uint64_t)s.NF * s.Fs, m->m_bf_qf0.p);
        to_bf16(m, s.yfeat, s.n_items, s.Fs, m->m_bf_yfeat.p);
        bf.ifeat = m->m_bf_ifeat.as<__nv_bfloat16>();
        bf.qf0 = m->m_bf_qf0.as<__nv_bfloat16>();
        bf.yfeat = m->m_bf_yfeat.as<__nv_bfloat16>();
    }
    if (prec >= TSVD_PREC_BF16_READ_ALL) {
        bf.ufeat = m->m_bf_ufeat.as<__nv_bfloat16>();
        bf.ufeat2 = m->m_bf_ufeat2.as<__nv_bfloat16>();
        bf.ycache = m->m_bf_ycache.as<__nv_bfloat16>();
    }
    const int vpl = (int)(s.Fs / 32);
    if (prec == TSVD_PREC_FP32) {
        TSVD_DISPATCH(vpl, (strat_launch<V, false, false>(m, p, bf)));
    } else if (prec == TSVD_PREC_BF16_READ) {
        TSVD_DISPATCH(vpl, (strat_launch<V, true, false>(m, p, bf)));
    } else {
        TSVD_DISPATCH(vpl, (strat_launch<V, true, true>(m, p, bf)));
    }
}

}  // namespace tsvd

// ---------------------------------------------------------------------------
// Fold-in and user reset entry points.
// ---------------------------------------------------------------------------
namespace {
thread_local std::string g_fold_err;

template <class F>
int fguard(tsvd_model* m, F&& f) {
    try {
        f();
        return TSVD_OK;
    } catch (const tsvd::Error& e) {
        if (m) m->err = e.what();
        g_fold_err = e.what();
        return e.status;
    } catch (const std::exception& e) {
        if (m) m->err = e.what();
        g_fold_err = e.what();
        return TSVD_ERR_INVALID;
    }
}
}  // namespace

extern "C" int tsvd_foldin(tsvd_model* m, const uint32_t* users, uint64_t n, uint32_t passes) {
    using namespace tsvd;
    if (!m || (!users && n)) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return fguard(m, [&] {
        if (n == 0 || passes == 0) return;
        if (n >= (1ull << 32)) throw Error(TSVD_ERR_INVALID, "too many users");
        for (uint64_t k = 0; k < n; ++k)
            if (users[k] >= m->d.n_users) throw Error(TSVD_ERR_INVALID, "user out of range");
        TSVD_CUDA(cudaSetDevice(m->device));
        DevMem du;
        du.alloc(n * 4);
        TSVD_CUDA(cudaMemcpyAsync(du.p, users, n * 4, cudaMemcpyHostToDevice, m->stream));
        if (!m->ycache_valid) {
            launch_rebuild_ycache(m);
        }
        EpochParams p = make_params(m);
        p.use_ycache = m->cfg.full_su ? 1 : 0;
        const int vpl = (int)(m->d.Fs / 32);
        for (uint32_t k = 0; k < passes; ++k) {
            TSVD_CUDA(cudaMemsetAsync(m->d.counters, 0, 64, m->stream));
            TSVD_DISPATCH(vpl, (foldin_launch<V>(m, p, du.as<uint32_t>(), (uint32_t)n)));
        }
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

extern "C" int tsvd_reset_users(tsvd_model* m, const uint32_t* users, uint64_t n, uint64_t seed) {
    using namespace tsvd;
    if (!m || (!users && n)) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return fguard(m, [&] {
        if (n == 0) return;
        for (uint64_t k = 0; k < n; ++k)
            if (users[k] >= m->d.n_users) throw Error(TSVD_ERR_INVALID, "user out of range");
        TSVD_CUDA(cudaSetDevice(m->device));
        const uint32_t Fs = m->d.Fs, F = m->d.F;
        std::vector<float> h((size_t)n * Fs, 0.0f);
        ChaCha12Stream g(seed);
        fill_normal_rows(g, m->cfg.sigma_u, n, F, h.data(), Fs);
        DevMem du, dp;
        du.alloc(n * 4);
        dp.alloc(h.size() * 4);
        TSVD_CUDA(cudaMemcpyAsync(du.p, users, n * 4, cudaMemcpyHostToDevice, m->stream));
        TSVD_CUDA(cudaMemcpyAsync(dp.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, m->stream));
        k_reset_users<<<(unsigned)n, 128, 0, m->stream>>>(m->d, du.as<uint32_t>(), (uint32_t)n, dp.as<float>());
        TSVD_CUDA(cudaGetLastError());
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}
