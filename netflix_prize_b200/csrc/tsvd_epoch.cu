// Epoch kernels of the tsvdx4 factorizer (TxModel::fit_epoch,
// src/tx.rs:734-1115, tx4 mode with low_memory = true).
//
// Work unit = one user (user stratum) or one item (item stratum), one warp
// each; a feature row of Fs floats lives in registers as VPL = Fs / 32 values
// per lane, and row dot products are warp butterfly reductions.
//
// Schedules
//  HOGWILD     the reference's per-user pass (su gather, sequential ratings,
//              y update at the end of the user) with all users of an epoch
//              in flight at once; item rows are read and written in place.
//  STRATIFIED  the reference's parallel schedule (src/tsvdx4p.rs:390-805):
//              user stratum with frozen item tables (no conflicts), NSVD1
//              deltas reduced per item in by-item order, ycache rebuild,
//              item stratum with frozen user tables. Deterministic.
#include <cstring>

#include "rand_stream.hpp"
#include "tsvd_device.cuh"

namespace tsvd {
namespace {

constexpr int kWarps = 8;  // warps per block
constexpr int kThreads = kWarps * 32;

struct EpochParams {
    float lr_u, lr_u2, lr_ub, lr_ubd, lr_i, lr_ib, lr_y, lr_yb, lr_tu, lr_ti, lr_ta, lr_ibf, lr_iqf, lr_cu;
    float reg_iqf, reg_cu, reg_u, reg_u2, reg_i, reg_y;
    float w_bias, w_factor;
    float nsvd_norm_exp;
    int32_t sum_err_bug;
    int32_t full_su;
    int32_t use_ycache;  // su of a user equals ycache[u] (stratified, full_su, ycache valid)
};

EpochParams make_params(const tsvd_model* m) {
    const tsvd_config& c = m->cfg;
    EpochParams p;
    p.lr_u = c.lr_u; p.lr_u2 = c.lr_u2; p.lr_ub = c.lr_ub; p.lr_ubd = c.lr_ubd; p.lr_i = c.lr_i;
    p.lr_ib = c.lr_ib; p.lr_y = c.lr_y; p.lr_yb = c.lr_yb; p.lr_tu = c.lr_tu; p.lr_ti = c.lr_ti;
    p.lr_ta = c.lr_ta; p.lr_ibf = c.lr_ibf; p.lr_iqf = c.lr_iqf; p.lr_cu = c.lr_cu;
    p.reg_iqf = c.reg_iqf; p.reg_cu = c.reg_cu; p.reg_u = c.reg_u; p.reg_u2 = c.reg_u2; p.reg_i = c.reg_i;
    p.reg_y = c.reg_y;
    p.w_bias = c.w_bias; p.w_factor = c.w_factor;
    p.nsvd_norm_exp = m->opts.nsvd_norm_exp;
    p.sum_err_bug = c.sum_err_bug;
    p.full_su = c.full_su;
    p.use_ycache = 0;
    return p;
}

// Sum of y rows (and ybias) over `n` items produced by `item_of(k)`, in order.
template <int VPL, class ItemOf>
__device__ __forceinline__ void gather_y(const DeviceState& s, uint64_t n, ItemOf item_of, int lane, float (&su)[VPL],
                                         float& sub) {
    for (uint64_t base = 0; base < n; base += 32) {
        const uint32_t cnt = (uint32_t)(n - base < 32 ? n - base : 32);
        const uint32_t mine = lane < (int)cnt ? item_of(base + lane) : 0u;
#pragma unroll 4
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t it = __shfl_sync(kFull, mine, j);
            float y[VPL];
            Row<VPL>::load_cg(s.yfeat + (size_t)it * s.Fs, lane, y);
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] += y[v];
            sub += __ldcg(s.ybias + it);
        }
    }
}

// ---------------------------------------------------------------------------
// User stratum (both schedules).
// ---------------------------------------------------------------------------
template <int VPL, bool HOG>
__global__ void __launch_bounds__(kThreads) k_user_pass(DeviceState s, EpochParams p, const uint32_t* __restrict__ order,
                                                        uint32_t n_work) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    (void)NF;
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

        // ---- NSVD1 user sum su = |N(u)|^-1/2 sum_j y_j (src/tx.rs:800-822)
        float su[VPL], sub;
        if (!HOG && p.use_ycache) {
            Row<VPL>::load_cg(s.ycache + (size_t)u * Fs, lane, su);
            sub = __ldcg(s.ycache_bias + u);
        } else {
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = 0.0f;
            sub = 0.0f;
            const Rec* rr = s.rec + start;
            gather_y<VPL>(s, end - start, [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su, sub);
            if (p.full_su) {
                const uint32_t* pp = s.pr_item + ps;
                gather_y<VPL>(s, pe - ps, [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sub);
            }
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = su[v] / norm;
            sub = sub / norm;
            Row<VPL>::store(s.ycache + (size_t)u * Fs, lane, su);
            if (lane == 0) s.ycache_bias[u] = sub;
        }

        // ---- user state in registers
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
            // software pipeline: rows of rating j+1 are requested before rating j is used
            float qn[VPL], qfn[VPL];
            {
                const Rec r0 = shfl_rec(mine, 0);
                const uint32_t i0 = rec_id(r0.key);
                if (HOG) {
                    Row<VPL>::load_cg(s.ifeat + (size_t)i0 * Fs, lane, qn);
                    Row<VPL>::load_cg(s.ifeat_freq + (size_t)i0 * NF * Fs, lane, qfn);
                } else {
                    Row<VPL>::load_nc(s.ifeat + (size_t)i0 * Fs, lane, qn);
                    Row<VPL>::load_nc(s.ifeat_freq + (size_t)i0 * NF * Fs, lane, qfn);
                }
            }
            for (uint32_t j = 0; j < cnt; ++j) {
                const Rec r = shfl_rec(mine, j);
                const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
                float q[VPL], qf[VPL];
#pragma unroll
                for (int v = 0; v < VPL; ++v) { q[v] = qn[v]; qf[v] = qfn[v]; }
                const Rec rn = shfl_rec(mine, j + 1 < cnt ? j + 1 : j);
                if (j + 1 < cnt) {
                    const uint32_t in = rec_id(rn.key);
                    if (HOG) {
                        Row<VPL>::load_cg(s.ifeat + (size_t)in * Fs, lane, qn);
                        Row<VPL>::load_cg(s.ifeat_freq + (size_t)in * NF * Fs, lane, qfn);
                    } else {
                        Row<VPL>::load_nc(s.ifeat + (size_t)in * Fs, lane, qn);
                        Row<VPL>::load_nc(s.ifeat_freq + (size_t)in * NF * Fs, lane, qfn);
                    }
                }
                // low_memory: the frequency bin used in training is always 0 (src/tx.rs:834,873)
                const float ib = HOG ? __ldcg(s.ibias + i) : __ldg(s.ibias + i);
                const float bit = HOG ? __ldcg(s.bit_bin + (size_t)i * T + tb) : __ldg(s.bit_bin + (size_t)i * T + tb);
                const float ibf = HOG ? __ldcg(s.ibias_freq + (size_t)i * NF) : __ldg(s.ibias_freq + (size_t)i * NF);
                float bud = 0.0f;
                const bool hud = r.ud < s.n_ud;
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
                const float score = gb + bu_t + bi_t * cu_t + dot;
                const float err = score - r.res;
                const float err_b = HOG ? err * p.w_bias : err;
                const float err_d = HOG ? err * p.w_factor : err;

                ub -= p.lr_ub * err_b;
                {
                    const float nb = but - p.lr_tu * err_b;
                    if (lane == (int)(tb & 31)) {
                        if (tb < 32) bb0 = nb;
                        else bb1 = nb;
                    }
                }
                al -= p.lr_ta * err_b * dv;
                if (lane == 0 && hud) s.ubias_day[r.ud] = bud - p.lr_ubd * err_b;
                if (HOG && lane == 0) {
                    __stcg(s.ibias + i, ib - p.lr_ib * (err_b * cu_t));
                    __stcg(s.bit_bin + (size_t)i * T + tb, bit - p.lr_ti * (err_b * cu_t));
                    __stcg(s.ibias_freq + (size_t)i * NF, ibf - p.lr_ibf * (err_b * cu_t));
                }
                cuu -= p.lr_cu * (err_b * bi_t + p.reg_cu * (cuu - 1.0f));
                if (!p.sum_err_bug) sum_err += err_b;
                else
                    for (uint32_t kk = 0; kk < s.F; ++kk) sum_err += err_b;
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    const float qe = q[v] + qf[v];
                    const float pk = pu[v], p2k = p2[v];
                    seq[v] += err_d * qe;
                    pu[v] = pk - p.lr_u * (err_d * qe + p.reg_u * pk);
                    p2[v] = p2k - p.lr_u2 * (err_d * qe * dv + p.reg_u2 * p2k);
                    if (HOG) {
                        const float pe = pk + dv * p2k + 0.0f + su[v];
                        q[v] = q[v] - p.lr_i * (err_d * pe + p.reg_i * q[v]);
                        qf[v] = qf[v] - p.lr_iqf * (err_d * pe + p.reg_iqf * qf[v]);
                    }
                }
                if (HOG) {
                    Row<VPL>::store(s.ifeat + (size_t)i * Fs, lane, q);
                    Row<VPL>::store(s.ifeat_freq + (size_t)i * NF * Fs, lane, qf);
                }
            }
        }
        // ---- write back user state
        Row<VPL>::store(s.ufeat + (size_t)u * Fs, lane, pu);
        Row<VPL>::store(s.ufeat2 + (size_t)u * Fs, lane, p2);
        if (lane == 0) {
            s.ubias[u] = ub;
            s.alpha_u[u] = al;
            s.cu[u] = cuu;
        }
        if (lane < (int)T) s.but_bin[(size_t)u * T + lane] = bb0;
        if (lane + 32 < (int)T) s.but_bin[(size_t)u * T + 32 + lane] = bb1;

        if (HOG) {
            // NSVD1 factor & bias updates at the end of the user (src/tx.rs:1099-1106)
            float g[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) g[v] = seq[v] / norm;
            const float eb = sum_err / norm;
            for (uint64_t base = start; base < end; base += 32) {
                const uint32_t cnt = (uint32_t)(end - base < 32 ? end - base : 32);
                const uint32_t mine = lane < (int)cnt ? rec_id(__ldg(&s.rec[base + lane].key)) : 0u;
                for (uint32_t j = 0; j < cnt; ++j) {
                    const uint32_t it = __shfl_sync(kFull, mine, j);
                    float y[VPL];
                    Row<VPL>::load_cg(s.yfeat + (size_t)it * Fs, lane, y);
#pragma unroll
                    for (int v = 0; v < VPL; ++v) y[v] = y[v] - p.lr_y * (g[v] + p.reg_y * y[v]);
                    Row<VPL>::store(s.yfeat + (size_t)it * Fs, lane, y);
                    if (lane == 0) __stcg(s.ybias + it, __ldcg(s.ybias + it) - p.lr_yb * eb);
                }
            }
        } else {
            float g[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) g[v] = seq[v] / norm;
            Row<VPL>::store(s.g_user + (size_t)u * Fs, lane, g);
            if (lane == 0) s.e_user[u] = sum_err / norm;
        }
    }
}

// ---------------------------------------------------------------------------
// Stratified: apply the NSVD1 deltas per item (apply_nsvd_deltas,
// src/tsvdx4p.rs:341-385). The per-item sum over the item's users runs in two
// fixed-order levels: fixed chunks of kChunkUsers consecutive by-item entries
// are summed by one warp each (k_y_partial), then each item adds its chunk
// partials in chunk order (k_y_combine). Same result on every run.
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
                    const uint32_t jj = j + q < cnt ? j + q : cnt - 1;
                    const uint32_t u = __shfl_sync(kFull, mine, jj);
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
// ycache[u] = |N(u)|^-1/2 sum over train and pr items (rebuild_ycache,
// src/tx.rs:391-418): train items in rating order, then pr items in pr order.
// ---------------------------------------------------------------------------
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_rebuild_ycache(DeviceState s) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * kWarps;
    for (uint32_t u = blockIdx.x * kWarps + (threadIdx.x >> 5); u < s.n_users; u += warps) {
        float su[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) su[v] = 0.0f;
        float sub = 0.0f;
        const uint64_t a = s.user_off[u], b = s.user_off[u + 1];
        const uint64_t pa = s.pr_off[u], pb = s.pr_off[u + 1];
        const Rec* rr = s.rec + a;
        gather_y<VPL>(s, b - a, [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su, sub);
        const uint32_t* pp = s.pr_item + pa;
        gather_y<VPL>(s, pb - pa, [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sub);
        const int32_t cnt = s.user_cnt_tr[u] + s.user_cnt_pr[u];
        if (cnt > 0) {
            const float nrm = sqrtf((float)cnt);
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = su[v] / nrm;
            sub = sub / nrm;
        }
        Row<VPL>::store(s.ycache + (size_t)u * s.Fs, lane, su);
        if (lane == 0) s.ycache_bias[u] = sub;
    }
}

// ---------------------------------------------------------------------------
// Stratified item stratum (fit_epoch_item, src/tsvdx4p.rs:644-762): items in
// parallel, each item's ratings in by-item order with the user tables frozen.
//
// An item's ratings form a serial chain (every update feeds the next dot
// product), and the most-rated items carry ~0.5% of all ratings each, so the
// chain of the hottest item bounds the pass. Items with >= kHeavy ratings get a
// whole CTA, warp-specialised: warps 1..7 gather the user rows of the next
// round of kRound ratings from HBM and fold them into
// pe = (p_u + ycache_u) + dev * p2_u plus the rating's bias scalars in shared
// memory (double-buffered rounds, one __syncthreads per round), while warp 0
// runs the chain from shared memory only. Lighter items take one warp each,
// with the next rating's rows prefetched into registers.
// ---------------------------------------------------------------------------
constexpr uint32_t kHeavy = 1024;
constexpr int kRound = 32;  // ratings per buffered round

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

template <int VPL>
__device__ void item_light(const DeviceState& s, const EpochParams& p, uint32_t i, int lane) {
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
        {
            const uint32_t u0 = rec_id(__shfl_sync(kFull, mine.key, 0));
            Row<VPL>::load_nc(s.ufeat + (size_t)u0 * Fs, lane, pn);
            Row<VPL>::load_nc(s.ufeat2 + (size_t)u0 * Fs, lane, p2n);
            Row<VPL>::load_nc(s.ycache + (size_t)u0 * Fs, lane, ycn);
        }
        for (uint32_t j = 0; j < cnt; ++j) {
            const Rec r = shfl_rec(mine, j);
            float pe[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) pe[v] = (pn[v] + ycn[v]) + r.dev * p2n[v];
            if (j + 1 < cnt) {
                const uint32_t un = rec_id(__shfl_sync(kFull, mine.key, j + 1));
                Row<VPL>::load_nc(s.ufeat + (size_t)un * Fs, lane, pn);
                Row<VPL>::load_nc(s.ufeat2 + (size_t)un * Fs, lane, p2n);
                Row<VPL>::load_nc(s.ycache + (size_t)un * Fs, lane, ycn);
            }
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

template <int VPL>
__global__ void __launch_bounds__(kThreads) k_item_pass(DeviceState s, EpochParams p) {
    extern __shared__ float smem[];
    __shared__ uint32_t sh_k;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t Fs = s.Fs, NF = s.NF;
    const uint32_t stride = Fs + 4;  // one staged rating: pe row + {bu_t, cu_t, res, key}
    float* qfs = smem;                                   // [NF][Fs]
    float* buf = smem + (size_t)NF * Fs;                 // [2][kRound][stride]
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
            if (warp == 0) item_light<VPL>(s, p, i, lane);
            for (;;) {
                uint32_t k2 = 0;
                if (lane == 0) k2 = atomicAdd(&s.counters[2], 1u);
                k2 = __shfl_sync(kFull, k2, 0);
                if (k2 >= s.n_items) return;
                item_light<VPL>(s, p, s.item_work[k2], lane);
            }
        }
        // ---------------- heavy item: whole CTA ----------------
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            qfs[e] = __ldcg(s.ifeat_freq + (size_t)i * NF * Fs + e);
        const uint64_t n = b - a;
        const uint32_t rounds = (uint32_t)((n + kRound - 1) / kRound);
        float q[VPL];
        ItemState st{};
        if (warp == 0) {
            Row<VPL>::load_cg(s.ifeat + (size_t)i * Fs, lane, q);
            st = load_item_state(s, i, lane);
        }
        // producers fill round r into buffer r & 1
        auto produce = [&](uint32_t r) {
            float* dst = buf + (size_t)(r & 1) * kRound * stride;
            const uint64_t r0 = a + (uint64_t)r * kRound;
            const uint64_t left = n - (uint64_t)r * kRound;
            const uint32_t m = (uint32_t)(left < (uint64_t)kRound ? left : (uint64_t)kRound);
            for (uint32_t j = warp - 1; j < m; j += kWarps - 1) {
                const Rec rr = load_rec(s.irec + r0 + j);
                const uint32_t u = rec_id(rr.key);
                float pu[VPL], p2[VPL], yc[VPL], pe[VPL];
                Row<VPL>::load_nc(s.ufeat + (size_t)u * Fs, lane, pu);
                Row<VPL>::load_nc(s.ufeat2 + (size_t)u * Fs, lane, p2);
                Row<VPL>::load_nc(s.ycache + (size_t)u * Fs, lane, yc);
                float bu_t, cu_t;
                user_scalars(s, rr, bu_t, cu_t);
#pragma unroll
                for (int v = 0; v < VPL; ++v) pe[v] = (pu[v] + yc[v]) + rr.dev * p2[v];
                float* row = dst + (size_t)j * stride;
#pragma unroll
                for (int v = 0; v < VPL; ++v) row[Row<VPL>::elem(lane, v)] = pe[v];
                if (lane == 0) {
                    row[Fs] = bu_t;
                    row[Fs + 1] = cu_t;
                    row[Fs + 2] = rr.res;
                    row[Fs + 3] = __uint_as_float(rr.key);
                }
            }
        };
        if (warp > 0) produce(0);
        __syncthreads();
        const float gb = s.gbias;
        for (uint32_t r = 0; r < rounds; ++r) {
            if (warp > 0) {
                if (r + 1 < rounds) produce(r + 1);
            } else {
                const float* src = buf + (size_t)(r & 1) * kRound * stride;
                const uint64_t left = n - (uint64_t)r * kRound;
                const uint32_t m = (uint32_t)(left < (uint64_t)kRound ? left : (uint64_t)kRound);
                for (uint32_t j = 0; j < m; ++j) {
                    const float* row = src + (size_t)j * stride;
                    float pe[VPL];
#pragma unroll
                    for (int v = 0; v < VPL; ++v) pe[v] = row[Row<VPL>::elem(lane, v)];
                    const float bu_t = row[Fs], cu_t = row[Fs + 1], res = row[Fs + 2];
                    const uint32_t key = __float_as_uint(row[Fs + 3]);
                    const uint32_t tb = rec_tbin(key), fb = rec_fbin(key);
                    float* qrow = qfs + (size_t)fb * Fs;
                    item_step<VPL>(p, gb, q, [&](int v) -> float& { return qrow[Row<VPL>::elem(lane, v)]; }, pe,
                                   bu_t, cu_t, res, tb, fb, lane, st);
                }
            }
            __syncthreads();
        }
        if (warp == 0) {
            Row<VPL>::store(s.ifeat + (size_t)i * Fs, lane, q);
            store_item_state(s, i, lane, st);
        }
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            __stcg(s.ifeat_freq + (size_t)i * NF * Fs + e, qfs[e]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <class K>
unsigned persistent_grid(K kernel, size_t smem) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return (unsigned)(sms * per_sm);
}

template <int VPL>
void launch_user_pass(tsvd_model* m, const EpochParams& p, const uint32_t* order, bool hog) {
    if (hog) {
        unsigned g = persistent_grid(k_user_pass<VPL, true>, 0);
        k_user_pass<VPL, true><<<g, kThreads, 0, m->stream>>>(m->d, p, order, m->d.n_users);
    } else {
        unsigned g = persistent_grid(k_user_pass<VPL, false>, 0);
        k_user_pass<VPL, false><<<g, kThreads, 0, m->stream>>>(m->d, p, order, m->d.n_users);
    }
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL>
void launch_y_apply(tsvd_model* m, const EpochParams& p) {
    unsigned g = persistent_grid(k_y_partial<VPL>, 0);
    k_y_partial<VPL><<<g, kThreads, 0, m->stream>>>(m->d);
    TSVD_CUDA(cudaGetLastError());
    unsigned g2 = ceil_div(m->d.n_items, kWarps);
    k_y_combine<VPL><<<g2, kThreads, 0, m->stream>>>(m->d, p);
    TSVD_CUDA(cudaGetLastError());
    m->launches += 2;
}

template <int VPL>
void launch_rebuild(tsvd_model* m) {
    unsigned g = persistent_grid(k_rebuild_ycache<VPL>, 0);
    k_rebuild_ycache<VPL><<<g, kThreads, 0, m->stream>>>(m->d);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL>
void launch_item_pass(tsvd_model* m, const EpochParams& p) {
    size_t smem = ((size_t)m->d.NF * m->d.Fs + 2ull * kRound * (m->d.Fs + 4)) * sizeof(float);
    TSVD_CUDA(cudaFuncSetAttribute(k_item_pass<VPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    unsigned g = persistent_grid(k_item_pass<VPL>, smem);
    k_item_pass<VPL><<<g, kThreads, smem, m->stream>>>(m->d, p);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
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

void reset_counters(tsvd_model* m) {
    TSVD_CUDA(cudaMemsetAsync(m->d.counters, 0, 64, m->stream));
}

}  // namespace

void rebuild_ycache(tsvd_model* m) {
    ProfScope ps(m, "rebuild_ycache");
    const int vpl = (int)(m->d.Fs / 32);
    TSVD_DISPATCH(vpl, launch_rebuild<V>(m));
    m->ycache_valid = true;
}

void run_epoch(tsvd_model* m, uint64_t epoch) {
    const tsvd_config& c = m->cfg;
    const int vpl = (int)(m->d.Fs / 32);
    EpochParams p = make_params(m);
    if (epoch == c.reset_u_epoch) {
        TSVD_CUDA(cudaMemsetAsync(m->d.ufeat, 0, m->m_ufeat.bytes, m->stream));
        TSVD_CUDA(cudaMemsetAsync(m->d.ufeat2, 0, m->m_ufeat2.bytes, m->stream));
    }
    reset_counters(m);
    if (m->opts.schedule == TSVD_SCHED_HOGWILD) {
        // per-epoch user order: injected, or get_users (src/lib.rs:486-494)
        std::vector<uint32_t> order;
        auto it = m->injected_order.find(epoch);
        if (it != m->injected_order.end()) order = it->second;
        else order = user_order(m->d.n_users, c.shuffle_users != 0, c.seed, epoch);
        TSVD_CUDA(cudaMemcpyAsync(m->m_perm.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));  // `order` leaves scope
        {
            ProfScope ps(m, "user_pass_hogwild");
            TSVD_DISPATCH(vpl, launch_user_pass<V>(m, p, m->m_perm.as<uint32_t>(), true));
        }
        rebuild_ycache(m);
    } else {
        p.use_ycache = (c.full_su && m->ycache_valid) ? 1 : 0;
        {
            ProfScope ps(m, "user_pass_stratified");
            TSVD_DISPATCH(vpl, launch_user_pass<V>(m, p, m->d.user_work, false));
        }
        {
            ProfScope ps(m, "y_apply");
            TSVD_DISPATCH(vpl, launch_y_apply<V>(m, p));
        }
        rebuild_ycache(m);
        {
            ProfScope ps(m, "item_pass");
            TSVD_DISPATCH(vpl, launch_item_pass<V>(m, p));
        }
    }
}

}  // namespace tsvd
