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
#include <algorithm>
#include <functional>
#include <mutex>
#include <numeric>
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

// The item rows a user-stratum rating reads: q_i and q^f_i of frequency bin fb.
// qe0 = q_i + q^f_{i,0}: with low_memory the user stratum trains frequency bin
// 0 only (src/tsvdx4p.rs:504-531) and reads the two rows only as this sum.
__global__ void k_make_qe0(const float* __restrict__ ifeat, const float* __restrict__ ifeat_freq, uint64_t rows,
                           uint32_t Fs, uint32_t NF, float* __restrict__ qe0) {
    const uint64_t n = rows * Fs;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = e / Fs, c = e - r * Fs;
        qe0[e] = ifeat[e] + ifeat_freq[r * NF * Fs + c];
    }
}

void make_qe0(tsvd_model* m);


template <int VPL, bool BF>
__device__ __forceinline__ void item_rows(const DeviceState& s, const Bf16Copies& bf, uint32_t i, uint32_t fb, int lane,
                                          float (&q)[VPL], float (&qf)[VPL]) {
    if constexpr (BF) {
        row_load_bf16<VPL>(bf.ifeat + (size_t)i * s.Fs, lane, q);
        row_load_bf16<VPL>(bf.qf0 + (size_t)i * s.Fs, lane, qf);  // BF16 copies: low_memory, bin 0
    } else {
        Row<VPL>::load_nc(s.ifeat + (size_t)i * s.Fs, lane, q);
        Row<VPL>::load_nc(s.ifeat_freq + ((size_t)i * s.NF + fb) * s.Fs, lane, qf);
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

// The ordinal head's thresholds (lane-uniform); lr_t = 0 in every stratified
// epoch, so they are constant within it.
__device__ __forceinline__ void load_thresholds(const DeviceState& s, float (&th)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) th[k] = s.raw ? __ldg(s.thresholds + k) : 0.0f;
}

// err of a rating: score - residual, or with the ordinal head the gradient of
// -log P(y) in the score (src/tx.rs:963-972); `target` is then the raw rating.
__device__ __forceinline__ float rating_err(const DeviceState& s, const float (&th)[4], float score, float target) {
    return s.raw ? ordinal_grad(th, score, (int)target) : score - target;
}

// Fixed-point accumulation of a per-day NSVD1 delta row (red.global.add.u64).
template <int VPL>
__device__ __forceinline__ void dyd_add(unsigned long long* row, int lane, const float (&x)[VPL]) {
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
        const long long q = __double2ll_rn((double)x[v] * kDydScale);
        atomicAdd(row + Row<VPL>::elem(lane, v), (unsigned long long)q);
    }
}

// ---------------------------------------------------------------------------
// User stratum (fit_epoch_user, src/tsvdx4p.rs:390-639). Item tables are
// read-only here; the item rows of rating j+1 are requested before rating j
// is used. With DAY (low_memory = false) each run of equal dates gets its
// su_day from yfeat_day (the run's training items, then the day's pr items,
// :500-527), the ratings add ufeat_day and su_day to p_u(t), ufeat_day is
// trained (:604-611), and at the run's end its error sum over
// sqrt(day count) goes to every item of the run as a yfeat_day delta
// (:614-622).
// ---------------------------------------------------------------------------
// MINB blocks per SM. Three (a few registers spilled) pay off where the pass
// is bound by its total work rather than by its longest user chains, which
// every extra resident warp slows: 26.2 -> 24.2 ms at the full shape, f = 256,
// but 10.0 -> 12.2 ms on 120,000 users with the same most active users.
template <int VPL, bool BF, bool DAY, int MINB = 2>
__global__ void __launch_bounds__(kThreads, MINB) k_user_strat(DeviceState s, EpochParams p, Bf16Copies bf,
                                                         const uint32_t* __restrict__ order, uint32_t n_work) {
    // FP32 with low_memory: the rating's item rows are read as their sum qe0
    constexpr bool QE = !BF && !DAY;
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    float th[4];
    load_thresholds(s, th);
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
        // the current run of equal dates (DAY)
        float sud[DAY ? VPL : 1], seqd[DAY ? VPL : 1], pud[DAY ? VPL : 1];
        float norm_day = 1.0f;
        uint64_t run0 = 0, run1 = 0;

        for (uint64_t base = start; base < end; base += 32) {
            const uint32_t cnt = (uint32_t)(end - base < 32 ? end - base : 32);
            Rec mine{};
            if (lane < (int)cnt) mine = load_rec(s.rec + base + lane);
            float qn[VPL], qfn[QE ? 1 : VPL];
            auto fetch_item = [&](uint32_t key) {
                if constexpr (QE) Row<VPL>::load_nc(s.qe0 + (size_t)rec_id(key) * Fs, lane, qn);
                else item_rows<VPL, BF>(s, bf, rec_id(key), DAY ? rec_fbin(key) : 0u, lane, qn, qfn);
            };
            fetch_item(__shfl_sync(kFull, mine.key, 0));
            for (uint32_t j = 0; j < cnt; ++j) {
                const Rec r = shfl_rec(mine, j);
                const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
                // low_memory: training uses frequency bin 0 (src/tsvdx4p.rs:504-531);
                // with the per-day terms, the run's bin
                const uint32_t fb = DAY ? rec_fbin(r.key) : 0u;
                const bool hud = r.ud < s.n_ud;
                const uint64_t t = base + j;
                if constexpr (DAY) {
                    if (t == start || t > run1) {
                        // a new run of equal dates (day_ranges, src/tx.rs:92-104)
                        run0 = run1 = t;
                        while (run1 + 1 < end && __ldg(&s.rec[run1 + 1].ud) == r.ud) ++run1;
#pragma unroll
                        for (int v = 0; v < VPL; ++v) sud[v] = seqd[v] = 0.0f;
                        float dummy = 0.0f;
                        gather_rows8<VPL>(s.yfeat_day, nullptr, Fs, run1 - run0 + 1,
                                          [&](uint64_t q) { return rec_id(__ldg(&s.rec[run0 + q].key)); }, lane, sud,
                                          dummy);
                        float day_cnt = (float)(run1 - run0 + 1);
                        if (p.full_su && hud) {
                            const uint64_t off = s.ud_list_off[r.ud];
                            const uint32_t pc = s.ud_pr_cnt[r.ud];
                            gather_rows8<VPL>(s.yfeat_day, nullptr, Fs, pc,
                                              [&](uint64_t q) { return __ldg(s.ud_list_item + off + q); }, lane, sud,
                                              dummy);
                            for (uint32_t c = 0; c < pc; ++c) day_cnt += 1.0f;
                        }
                        norm_day = sqrtf(day_cnt);
#pragma unroll
                        for (int v = 0; v < VPL; ++v) sud[v] = sud[v] / norm_day;
                        if (p.has_ud && hud) Row<VPL>::load_cg(s.ufeat_day + (size_t)r.ud * Fs, lane, pud);
                        else
#pragma unroll
                            for (int v = 0; v < VPL; ++v) pud[v] = 0.0f;
                    }
                }
                float qe[VPL];  // q_i + q^f_{i,fb}
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    if constexpr (QE) qe[v] = qn[v];
                    else qe[v] = qn[v] + qfn[v];
                }
                if (j + 1 < cnt) fetch_item(__shfl_sync(kFull, mine.key, j + 1));
                const float ib = __ldg(s.ibias + i);
                const float bit = __ldg(s.bit_bin + (size_t)i * T + tb);
                const float ibf = __ldg(s.ibias_freq + (size_t)i * NF + fb);
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
                for (int v = 0; v < VPL; ++v) {
                    float pev = (pu[v] + su[v]) + dv * p2[v];
                    if constexpr (DAY) {
                        if (p.has_ud && hud) pev += pud[v];
                        pev += sud[v];
                    }
                    part += qe[v] * pev;
                }
                const float dot = warp_sum(part);
                const float err = rating_err(s, th, gb + bu_t + bi_t * cu_t + dot, r.res);
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
                    const float pk = pu[v], p2k = p2[v];
                    seq[v] += err * qe[v];
                    pu[v] = pk - p.lr_u * (err * qe[v] + p.reg_u * pk);
                    p2[v] = p2k - p.lr_u2 * (err * qe[v] * dv + p.reg_u2 * p2k);
                    if constexpr (DAY) {
                        seqd[v] += err * qe[v];
                        if (p.has_ud && hud) pud[v] = pud[v] - p.lr_ud * (err * qe[v] + p.reg_ud * pud[v]);
                    }
                }
                if constexpr (DAY) {
                    if (t == run1) {
                        // end of the run: ufeat_day back, and the run's yfeat_day
                        // delta to each of its items (src/tsvdx4p.rs:614-622)
                        if (p.has_ud && hud) Row<VPL>::store(s.ufeat_day + (size_t)r.ud * Fs, lane, pud);
                        float gd[VPL];
#pragma unroll
                        for (int v = 0; v < VPL; ++v) gd[v] = seqd[v] / norm_day;
                        for (uint64_t q2 = run0; q2 <= run1; ++q2)
                            dyd_add<VPL>(s.dyd_fix + (size_t)rec_id(__ldg(&s.rec[q2].key)) * Fs, lane, gd);
                    }
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
// Entries whose user lies outside [u_lo, u_hi) are left out (a user block; the
// full range otherwise). An item's entries are sorted by user, so the ones
// kept are contiguous and keep their order. With `accumulate` the block's
// partial is added to the chunk's earlier blocks' (blocks in user order), and
// chunks without entries in the block are left alone: passes over user blocks
// whose g_user rows fit in L2 gather from L2 instead of HBM.
template <int VPL>
// split (optional): per chunk, the first entry of each pass's user block
// (split[c * (passes + 1) + k]); without it the block's range is searched.
__global__ void __launch_bounds__(kThreads) k_y_partial(DeviceState s, uint32_t u_lo, uint32_t u_hi,
                                                        int accumulate, const uint64_t* __restrict__ split,
                                                        uint32_t passes, uint32_t pass) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs;
    constexpr int B = 8;  // rows in flight per warp
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&s.counters[1], 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= s.n_chunks) break;
        uint64_t a = s.chunk_lo[c];
        uint64_t b = s.chunk_lo[c + 1];
        if (b - a > kChunkUsers) b = a + kChunkUsers;
        if (split) {
            a = split[(size_t)c * (passes + 1) + pass];
            b = split[(size_t)c * (passes + 1) + pass + 1];
            if (accumulate && a == b) continue;
        } else if (u_lo != 0 || u_hi != 0xffffffffu) {
            // the chunk's entries of users u_lo..u_hi-1 (sorted by user)
            uint64_t lo = a, hi = b;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (rec_id(__ldg(&s.irec[mid].key)) < u_lo) lo = mid + 1;
                else hi = mid;
            }
            uint64_t lo2 = lo, hi2 = b;
            while (lo2 < hi2) {
                const uint64_t mid = (lo2 + hi2) >> 1;
                if (rec_id(__ldg(&s.irec[mid].key)) < u_hi) lo2 = mid + 1;
                else hi2 = mid;
            }
            a = lo;
            b = lo2;
            if (accumulate && a == b) continue;
        }
        // rows wider than 32 * VPL columns (n_feat > 256) in slices
        for (uint32_t c0 = 0; c0 < Fs; c0 += 32 * VPL) {
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
                        Row<VPL>::load_nc(s.g_user + (size_t)u * Fs + c0, lane, g[q]);
                        e[q] = c0 == 0 ? __ldg(s.e_user + u) : 0.0f;
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
            if (accumulate) {
                float prev[VPL];
                Row<VPL>::load_cg(s.chunk_part + (size_t)c * Fs + c0, lane, prev);
#pragma unroll
                for (int v = 0; v < VPL; ++v) acc[v] = prev[v] + acc[v];
                if (c0 == 0) eacc = __ldcg(s.chunk_epart + c) + eacc;
            }
            Row<VPL>::store(s.chunk_part + (size_t)c * Fs + c0, lane, acc);
            if (lane == 0 && c0 == 0) s.chunk_epart[c] = eacc;
        }
    }
}

// split[c * (nb) + k] = the first entry of chunk c whose user is >= bounds[k]
// (the chunk's entries are sorted by user).
__global__ void k_chunk_splits(DeviceState s, const uint32_t* __restrict__ bounds, uint32_t nb,
                               uint64_t* __restrict__ split) {
    const uint64_t n = (uint64_t)s.n_chunks * nb;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(e / nb), k = (uint32_t)(e % nb);
        uint64_t lo = s.chunk_lo[c], hi = s.chunk_lo[c + 1];
        if (hi - lo > kChunkUsers) hi = lo + kChunkUsers;
        const uint32_t u = bounds[k];
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (rec_id(__ldg(&s.irec[mid].key)) < u) lo = mid + 1;
            else hi = mid;
        }
        split[e] = lo;
    }
}

// The per-chunk split table for the user-block bounds `bounds`, made when the
// bounds change (outside a stream capture; inside one, a stale table gives
// null and the passes search instead).
const uint64_t* chunk_splits(tsvd_model* m, const DeviceState& s, const std::vector<uint32_t>& bounds) {
    if (bounds != m->h_split_bounds || !m->m_chunk_split.p) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        TSVD_CUDA(cudaStreamIsCapturing(m->stream, &cs));
        if (cs != cudaStreamCaptureStatusNone) return nullptr;
        const size_t n = (size_t)s.n_chunks * bounds.size();
        if (m->m_chunk_split.bytes < n * 8) m->m_chunk_split.alloc(n * 8);
        if (m->m_split_bounds.bytes < bounds.size() * 4) m->m_split_bounds.alloc(bounds.size() * 4);
        TSVD_CUDA(cudaMemcpyAsync(m->m_split_bounds.p, bounds.data(), bounds.size() * 4, cudaMemcpyHostToDevice,
                                  m->stream));
        const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
        k_chunk_splits<<<grid, 256, 0, m->stream>>>(s, m->m_split_bounds.as<uint32_t>(), (uint32_t)bounds.size(),
                                                    m->m_chunk_split.as<uint64_t>());
        TSVD_CUDA(cudaGetLastError());
        TSVD_CUDA(cudaStreamSynchronize(m->stream));  // `bounds` is the caller's
        m->launches++;
        m->h_split_bounds = bounds;
    }
    return m->m_chunk_split.as<uint64_t>();
}

// The NSVD1 delta sums of users u_lo..u_hi-1 into the chunk partials, in
// passes over user blocks of at most ~64 MB of g_user rows (L2 holds one).
// Each chunk's entries of a block come from a split table made once for the
// blocks' bounds, not from a search in every pass.
template <int VPL>
void y_partial_passes(tsvd_model* m, const DeviceState& s, uint32_t u_lo, uint32_t u_hi) {
    const uint64_t row_bytes = (uint64_t)s.Fs * 4;
    const uint32_t per = (uint32_t)std::max<uint64_t>(1, (64ull << 20) / row_bytes);
    const unsigned g = persistent_grid(k_y_partial<VPL>, 0);
    const bool whole = u_lo == 0 && u_hi >= s.n_users;
    std::vector<uint32_t> bounds;
    for (uint64_t b0 = u_lo; b0 < u_hi || b0 == u_lo; b0 += per) {
        bounds.push_back((uint32_t)b0);
        if (std::min<uint64_t>(u_hi, b0 + per) >= u_hi) break;
    }
    bounds.push_back(u_hi);
    const uint32_t passes = (uint32_t)bounds.size() - 1;
    const bool one = whole && passes == 1;  // a single pass over every user
    const uint64_t* split = one ? nullptr : chunk_splits(m, s, bounds);
    for (uint32_t k = 0; k < passes; ++k) {
        TSVD_CUDA(cudaMemsetAsync(s.counters + 1, 0, 4, m->stream));
        k_y_partial<VPL><<<g, kThreads, 0, m->stream>>>(s, one ? 0u : bounds[k], one ? 0xffffffffu : bounds[k + 1],
                                                        k == 0 ? 0 : 1, split, passes, k);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
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
        const float nc = (float)(s.item_off[i + 1] - s.item_off[i]);
        const float scale = p.nsvd_norm_exp == 0.0f ? 1.0f : powf(nc, p.nsvd_norm_exp);
        for (uint32_t x0 = 0; x0 < Fs; x0 += 32 * VPL) {
            float acc[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) acc[v] = 0.0f;
            for (uint32_t c = c0; c < c1; ++c) {
                float g[VPL];
                Row<VPL>::load_cg(s.chunk_part + (size_t)c * Fs + x0, lane, g);
#pragma unroll
                for (int v = 0; v < VPL; ++v) acc[v] += g[v];
            }
            float y[VPL];
            Row<VPL>::load_cg(s.yfeat + (size_t)i * Fs + x0, lane, y);
#pragma unroll
            for (int v = 0; v < VPL; ++v) y[v] = y[v] - p.lr_y * (acc[v] / scale + p.reg_y * y[v]);
            Row<VPL>::store(s.yfeat + (size_t)i * Fs + x0, lane, y);
            if (s.dyd_fix) {
                // per-day NSVD1 deltas, same divisor (src/tsvdx4p.rs:370-384)
                float yd[VPL];
                Row<VPL>::load_cg(s.yfeat_day + (size_t)i * Fs + x0, lane, yd);
                const unsigned long long* drow = s.dyd_fix + (size_t)i * Fs + x0;
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    const float d = (float)((double)(long long)__ldcg(drow + Row<VPL>::elem(lane, v)) / kDydScale);
                    yd[v] = yd[v] - p.lr_yd * (d / scale + p.reg_yd * yd[v]);
                }
                Row<VPL>::store(s.yfeat_day + (size_t)i * Fs + x0, lane, yd);
            }
        }
        float eacc = 0.0f;
        for (uint32_t c = c0; c < c1; ++c) eacc += __ldcg(s.chunk_epart + c);
        if (lane == 0) s.ybias[i] = s.ybias[i] - p.lr_yb * (eacc / scale);
    }
}

// A user block's NSVD1 delta sums per item (chunk partials added in chunk
// order) into sums [I, Fs] and sums_e [I], instead of applying them: the
// ranks of a sharded run add their blocks' sums before the apply.
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_y_block_sums(DeviceState s, float* __restrict__ sums,
                                                           float* __restrict__ sums_e) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs;
    const uint32_t warps = gridDim.x * kWarps;
    for (uint32_t i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < s.n_items; i += warps) {
        const uint32_t c0 = s.item_chunk0[i], c1 = s.item_chunk0[i + 1];
        for (uint32_t x0 = 0; x0 < Fs; x0 += 32 * VPL) {
            float acc[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) acc[v] = 0.0f;
            for (uint32_t c = c0; c < c1; ++c) {
                float g[VPL];
                Row<VPL>::load_cg(s.chunk_part + (size_t)c * Fs + x0, lane, g);
#pragma unroll
                for (int v = 0; v < VPL; ++v) acc[v] += g[v];
            }
            Row<VPL>::store(sums + (size_t)i * Fs + x0, lane, acc);
        }
        float eacc = 0.0f;
        for (uint32_t c = c0; c < c1; ++c) eacc += __ldcg(s.chunk_epart + c);
        if (lane == 0) sums_e[i] = eacc;
    }
}

// apply_nsvd_deltas (src/tsvdx4p.rs:341-385) of summed deltas: sums [I, Fs],
// sums_e [I] and, with the per-day terms, the fixed-point yfeat_day sums.
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_y_apply_sums(DeviceState s, EpochParams p,
                                                           const float* __restrict__ sums,
                                                           const float* __restrict__ sums_e,
                                                           const long long* __restrict__ dyd) {
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs;
    const uint32_t warps = gridDim.x * kWarps;
    for (uint32_t i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < s.n_items; i += warps) {
        const uint64_t ncnt = s.item_off[i + 1] - s.item_off[i];
        if (ncnt == 0) continue;
        const float scale = p.nsvd_norm_exp == 0.0f ? 1.0f : powf((float)ncnt, p.nsvd_norm_exp);
        for (uint32_t x0 = 0; x0 < Fs; x0 += 32 * VPL) {
            float acc[VPL], y[VPL];
            Row<VPL>::load_cg(sums + (size_t)i * Fs + x0, lane, acc);
            Row<VPL>::load_cg(s.yfeat + (size_t)i * Fs + x0, lane, y);
#pragma unroll
            for (int v = 0; v < VPL; ++v) y[v] = y[v] - p.lr_y * (acc[v] / scale + p.reg_y * y[v]);
            Row<VPL>::store(s.yfeat + (size_t)i * Fs + x0, lane, y);
            if (dyd) {
                float yd[VPL];
                Row<VPL>::load_cg(s.yfeat_day + (size_t)i * Fs + x0, lane, yd);
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    const float d = (float)((double)__ldcg(dyd + (size_t)i * Fs + x0 + Row<VPL>::elem(lane, v)) /
                                            kDydScale);
                    yd[v] = yd[v] - p.lr_yd * (d / scale + p.reg_yd * yd[v]);
                }
                Row<VPL>::store(s.yfeat_day + (size_t)i * Fs + x0, lane, yd);
            }
        }
        if (lane == 0) s.ybias[i] = s.ybias[i] - p.lr_yb * (__ldcg(sums_e + i) / scale);
    }
}

// ---------------------------------------------------------------------------
// Item stratum. An item's ratings form a serial chain (every update feeds the
// next dot product), and the most-rated items carry ~0.5% of all ratings
// each, so the chain of the hottest item bounds the pass. Items with at least
// s.heavy_min ratings (an option, 32768 by default) get a whole CTA of kCW + kPW warps, in rounds of kRound ratings:
//   producers (kPW warps) gather the next round's user rows into
//     pe = (p_u + ycache_u) + dev * p2_u plus the rating's bias scalars,
//     form the round's Gram matrix on the tensor cores and from it the
//     round's lower-triangular system (everything about the round that does
//     not depend on the item's current rows);
//   consumers (kCW warps, each owning every kCW-th 32-column stripe of q and
//     of the q^f rows) take the dots with the item's rows, warp 0 solves the
//     system for the round's errors, and all of them apply the closed-form
//     updates to their stripes.
// Rounds are double-buffered with one __syncthreads per round. Lighter items
// take one warp each, with the next rating's rows prefetched into registers.
// ---------------------------------------------------------------------------
constexpr int kRound = 32;  // ratings per buffered round
constexpr uint32_t kMS = kRound + 1;  // padded row stride of the round's system M
constexpr int kCW = 4;                // consumer warps
constexpr int kPW = 8;                // producer warps
constexpr int kItemThreads = (kCW + kPW) * 32;
constexpr int kVecs = 9;              // per-rating vectors of a round
// BF16 rows of the Gram operands: Fs values + 16 bytes, so that the eight
// 16-byte row segments an ldmatrix reads fall in distinct bank groups
__host__ __device__ constexpr uint32_t hl_pitch(uint32_t Fs) { return Fs * 2 + 16; }
static_assert(kPW * 4 == kRound, "each producer warp stages four of the round's ratings");

// Shared-memory layout of the item pass, in floats (every offset a multiple of 4).
struct ItemSmem {
    uint32_t qfs, qsh, buf, hl, mbuf, vec, pd, sv, ap, st, pw, total;
};
__host__ __device__ inline ItemSmem item_smem(uint32_t Fs, uint32_t NF) {
    ItemSmem L;
    uint32_t o = 0;
    L.qfs = o;  o += NF * (Fs + 4);             // the item's q^f rows, padded
    L.qsh = o;  o += Fs;                        // q at the round's start
    L.buf = o;  o += 2 * kRound * (Fs + 4);     // two rounds of pe rows + {bu_t, cu_t, res, key}
    L.hl = o;   o += 2 * kRound * (Fs / 2 + 4); // BF16 high and low parts of the produced round's pe rows
    L.mbuf = o; o += 2 * kRound * kMS;          // two rounds of the system M (row j: M_j,i)
    L.vec = o;  o += 2 * kVecs * kRound;        // two rounds of per-rating weights
    L.pd = o;   o += kCW * 2 * kRound;          // consumers' partial dots
    L.sv = o;   o += 4 * kRound;                // the round's update weights (q, q^f, biases)
    L.ap = o;   o += 4 * kRound;                // per rating {w_q, w_f, decay, bin | previous << 8}
    L.st = o;   o += 132;                       // the item's biases: ib, bit_bin[64], ibias_freq[64]
    L.pw = o;   o += 2 * 36;                    // a_i^n, a_f^n for n = 0..kRound
    L.total = o;
    return L;
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

// The user-side rows of a by-item rating: p_u + ycache_u and p2_u.
template <int VPL, bool BF>
__device__ __forceinline__ void pe_rows(const DeviceState& s, const Bf16Copies& bf, uint32_t u, int lane,
                                        float (&pyc)[VPL], float (&p2)[VPL]) {
    if constexpr (BF) {
        row_load_bf16<VPL>(bf.pyc + (size_t)u * s.Fs, lane, pyc);
        row_load_bf16<VPL>(bf.ufeat2 + (size_t)u * s.Fs, lane, p2);
    } else {
        Row<VPL>::load_nc(s.pyc + (size_t)u * s.Fs, lane, pyc);
        Row<VPL>::load_nc(s.ufeat2 + (size_t)u * s.Fs, lane, p2);
    }
}

// One SGD step of the item chain; qf_at(v) is this lane's v-th element of q^f[fb].
template <int VPL, class QF>
__device__ __forceinline__ void item_step(const DeviceState& s, const EpochParams& p, const float (&th)[4], float gb,
                                          float (&q)[VPL], QF&& qf_at, const float (&pe)[VPL], float bu_t,
                                          float cu_t, float res, uint32_t tb, uint32_t fb, int lane, ItemState& st) {
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
    const float err = rating_err(s, th, gb + bu_t + bi_t * cu_t + dot, res);
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

// One item by one warp (fit_epoch_item, src/tsvdx4p.rs:644-762). With DAY the
// ratings' p_u(t) also takes ufeat_day and ycache_day of the rating's day
// (:712-719), loaded a step ahead with the user rows.
template <int VPL, bool BF, bool DAY>
__device__ void item_light(const DeviceState& s, const EpochParams& p, const Bf16Copies& bf, uint32_t i, int lane) {
    const uint32_t Fs = s.Fs, NF = s.NF;
    const uint64_t a = s.item_off[i], b = s.item_off[i + 1];
    if (a == b) return;
    float th[4];
    load_thresholds(s, th);
    float q[VPL];
    Row<VPL>::load_cg(s.ifeat + (size_t)i * Fs, lane, q);
    ItemState st = load_item_state(s, i, lane);
    float* qf_base = s.ifeat_freq + (size_t)i * NF * Fs;
    const float gb = s.gbias;
    for (uint64_t base = a; base < b; base += 32) {
        const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
        // the chunk's records and user-side scalars, one rating per lane
        Rec mine{};
        float bu_l = 0.0f, cu_l = 0.0f;
        if (lane < (int)cnt) {
            mine = load_rec(s.irec + base + lane);
            user_scalars(s, mine, bu_l, cu_l);
        }
        float pn[VPL], p2n[VPL], dn[DAY ? VPL : 1], cn[DAY ? VPL : 1];
        auto fetch = [&](uint32_t j) {
            const uint32_t uj = rec_id(__shfl_sync(kFull, mine.key, j));
            pe_rows<VPL, BF>(s, bf, uj, lane, pn, p2n);
            if constexpr (DAY) {
                const uint32_t udj = __shfl_sync(kFull, mine.ud, j);
                if (udj < s.n_ud) {
                    Row<VPL>::load_nc(s.ufeat_day + (size_t)udj * Fs, lane, dn);
                    Row<VPL>::load_nc(s.ycache_day + (size_t)udj * Fs, lane, cn);
                }
            }
        };
        fetch(0);
        // the q^f row of the current rating's bin; the next rating's row is
        // loaded a step ahead when its bin differs (this rating leaves it alone)
        uint32_t fcur = rec_fbin(__shfl_sync(kFull, mine.key, 0));
        float qfv[VPL];
        Row<VPL>::load_cg(qf_base + (size_t)fcur * Fs, lane, qfv);
        for (uint32_t j = 0; j < cnt; ++j) {
            const Rec r = shfl_rec(mine, j);
            float pe[VPL];
#pragma unroll
            for (int v = 0; v < VPL; ++v) pe[v] = pn[v] + r.dev * p2n[v];
            if constexpr (DAY) {
                if (r.ud < s.n_ud) {
#pragma unroll
                    for (int v = 0; v < VPL; ++v) {
                        pe[v] += dn[v];
                        pe[v] += cn[v];
                    }
                }
            }
            if (j + 1 < cnt) fetch(j + 1);
            const float bu_t = __shfl_sync(kFull, bu_l, j), cu_t = __shfl_sync(kFull, cu_l, j);
            const uint32_t tb = rec_tbin(r.key), fb = fcur;
            const uint32_t fnext = j + 1 < cnt ? rec_fbin(__shfl_sync(kFull, mine.key, j + 1)) : fcur;
            float qfn[VPL];
            if (fnext != fcur) Row<VPL>::load_cg(qf_base + (size_t)fnext * Fs, lane, qfn);
            item_step<VPL>(s, p, th, gb, q, [&](int v) -> float& { return qfv[v]; }, pe, bu_t, cu_t, r.res, tb, fb,
                           lane, st);
            Row<VPL>::store(qf_base + (size_t)fcur * Fs, lane, qfv);
            if (fnext != fcur) {
#pragma unroll
                for (int v = 0; v < VPL; ++v) qfv[v] = qfn[v];
            }
            fcur = fnext;
        }
    }
    Row<VPL>::store(s.ifeat + (size_t)i * Fs, lane, q);
    store_item_state(s, i, lane, st);
}

// x = hi + lo + r with hi, lo in BF16 (round to nearest even), |r| <= 2^-17 |x|.
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// One staged rating: its FP32 pe row (for the consumers) and the BF16 high and
// low parts of it (the Gram operands), each element split once.
template <int VPL>
__device__ __forceinline__ void stage_row(float* row, uint8_t* hi_row, uint8_t* lo_row, int lane,
                                          const float (&pe)[VPL]) {
    if constexpr (VPL % 4 == 0) {
#pragma unroll
        for (int c = 0; c < VPL / 4; ++c) {
            const int col = c * 128 + lane * 4;
            const float4 x = make_float4(pe[4 * c], pe[4 * c + 1], pe[4 * c + 2], pe[4 * c + 3]);
            *reinterpret_cast<float4*>(row + col) = x;
            __nv_bfloat16 h[4], l[4];
            split_bf16(x.x, h[0], l[0]);
            split_bf16(x.y, h[1], l[1]);
            split_bf16(x.z, h[2], l[2]);
            split_bf16(x.w, h[3], l[3]);
            *reinterpret_cast<uint2*>(hi_row + 2 * col) = *reinterpret_cast<const uint2*>(h);
            *reinterpret_cast<uint2*>(lo_row + 2 * col) = *reinterpret_cast<const uint2*>(l);
        }
    } else {
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
            const int col = Row<VPL>::elem(lane, v);
            row[col] = pe[v];
            __nv_bfloat16 h, l;
            split_bf16(pe[v], h, l);
            reinterpret_cast<__nv_bfloat16*>(hi_row)[col] = h;
            reinterpret_cast<__nv_bfloat16*>(lo_row)[col] = l;
        }
    }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

// d (16x8, FP32) += a (16x16, BF16, row-major) . b (16x8, BF16, column-major)
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int VPL, bool BF, bool DAY>
__global__ void __launch_bounds__(kItemThreads, 1) k_item_pass(DeviceState s, EpochParams p, Bf16Copies bf) {
    extern __shared__ __align__(16) float smem[];
    __shared__ uint32_t sh_k;
    static_assert(kCW == 4, "the consumers' partial dots are summed as (0 + 1) + (2 + 3)");
    constexpr int CPL = (VPL + kCW - 1) / kCW;  // 32-column stripes per consumer warp
    constexpr int kChunk = 8;                   // ratings per step of the consumers' apply
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t Fs = s.Fs, NF = s.NF, T = s.T, NS = Fs / 32;
    const uint32_t stride = Fs + 4;  // one staged rating: pe row + {bu_t, cu_t, res, key}
    const uint32_t qs = Fs + 4;      // padded q^f row stride
    const ItemSmem L = item_smem(Fs, NF);
    float* qfs = smem + L.qfs;
    float* qsh = smem + L.qsh;
    float* buf = smem + L.buf;
    uint8_t* hl = reinterpret_cast<uint8_t*>(smem + L.hl);
    const uint32_t hp = hl_pitch(Fs);
    float* mbuf = smem + L.mbuf;
    float* vec = smem + L.vec;
    float* pd = smem + L.pd;
    float* sv = smem + L.sv;
    float4* ap = reinterpret_cast<float4*>(smem + L.ap);
    float* sst = smem + L.st;
    float* apow = smem + L.pw;  // apow[n] = a_i^n, fpow[n] = a_f^n (products in order)
    float* fpow = apow + 36;
    // update factors: x - lr (g + reg x) = a x - lr g
    const float a_i = 1.0f - p.lr_i * p.reg_i, a_f = 1.0f - p.lr_iqf * p.reg_iqf;
    if (threadIdx.x == 0) {
        float x = 1.0f, y = 1.0f;
        for (int e = 0; e <= kRound; ++e) {
            apow[e] = x;
            fpow[e] = y;
            x *= a_i;
            y *= a_f;
        }
    }
    const float gb = s.gbias;
    for (;;) {
        if (threadIdx.x == 0) sh_k = atomicAdd(&s.counters[2], 1u);
        __syncthreads();
        const uint32_t k = sh_k;
        __syncthreads();
        if (k >= s.n_item_work) return;
        const uint32_t i = s.item_work[k];
        const uint64_t a = s.item_off[i], b = s.item_off[i + 1];
        if (b - a < s.heavy_min) {
            // Items are ordered heaviest first: from here on every item is light.
            if (warp == 0) item_light<VPL, BF, DAY>(s, p, bf, i, lane);
            for (;;) {
                uint32_t k2 = 0;
                if (lane == 0) k2 = atomicAdd(&s.counters[2], 1u);
                k2 = __shfl_sync(kFull, k2, 0);
                if (k2 >= s.n_item_work) return;
                item_light<VPL, BF, DAY>(s, p, bf, s.item_work[k2], lane);
            }
        }
        // ---------------- heavy item: whole CTA ----------------
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            qfs[(e / Fs) * qs + e % Fs] = __ldcg(s.ifeat_freq + (size_t)i * NF * Fs + e);
        const uint64_t n = b - a;
        const uint32_t rounds = (uint32_t)((n + kRound - 1) / kRound);
        if (threadIdx.x < 64) {
            const uint32_t t = threadIdx.x;
            if (t == 0) sst[0] = __ldcg(s.ibias + i);
            sst[1 + t] = t < T ? __ldcg(s.bit_bin + (size_t)i * T + t) : 0.0f;
            sst[65 + t] = t < NF ? __ldcg(s.ibias_freq + (size_t)i * NF + t) : 0.0f;
        }
        float qv[CPL];  // consumer warp c: q columns 32 (c + kCW t) + lane
        if (warp < kCW) {
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const uint32_t sc = warp + kCW * t;
                qv[t] = sc < NS ? __ldcg(s.ifeat + (size_t)i * Fs + 32 * sc + lane) : 0.0f;
            }
        }
        auto round_len = [&](uint32_t r) -> uint32_t {
            const uint64_t left = n - (uint64_t)r * kRound;
            return (uint32_t)(left < (uint64_t)kRound ? left : (uint64_t)kRound);
        };
        // Producers load records two rounds ahead (one per lane) and the next
        // round's user scalars (on the lanes that stage them) a round ahead,
        // so that their latency overlaps the wait for the consumers.
        Rec rc1{}, rc2{};
        float us[7] = {};  // ubias, but_bin, alpha_u, ubias_day, ycache_bias, cu, cut
        // user rows (p_u + ycache_u, p2_u) of ratings pw and pw + 8 of the next
        // round, loaded at the end of the previous producer phase
        float px0[VPL], py0[VPL], px1[VPL], py1[VPL];
        auto fetch_rows0 = [&](uint32_t r) {  // rc1 holds round r's records
            const int pw = warp - kCW;
            const uint32_t m = round_len(r), j0 = pw, j1 = pw + kPW;
            const uint32_t u0 = rec_id(__shfl_sync(kFull, rc1.key, j0));
            const uint32_t u1 = rec_id(__shfl_sync(kFull, rc1.key, j1));
#pragma unroll
            for (int v = 0; v < VPL; ++v) px0[v] = py0[v] = px1[v] = py1[v] = 0.0f;
            if (j0 < m) pe_rows<VPL, BF>(s, bf, u0, lane, px0, py0);
            if (j1 < m) pe_rows<VPL, BF>(s, bf, u1, lane, px1, py1);
        };
        auto fetch_records = [&](uint32_t r, Rec& out) {
            out = Rec{};
            if (r < rounds && lane < (int)round_len(r)) out = load_rec(s.irec + a + (uint64_t)r * kRound + lane);
        };
        auto fetch_scalars = [&](uint32_t r) {  // rc1 holds round r's records
            const int pw = warp - kCW;
            if (lane < (int)round_len(r) && (lane & (kPW - 1)) == pw) {
                const uint32_t u = rec_id(rc1.key), tb = rec_tbin(rc1.key);
                const bool hud = rc1.ud < s.n_ud;
                us[0] = __ldg(s.ubias + u);
                us[1] = __ldg(s.but_bin + (size_t)u * s.T + tb);
                us[2] = __ldg(s.alpha_u + u);
                us[3] = hud ? __ldg(s.ubias_day + rc1.ud) : 0.0f;
                us[4] = __ldg(s.ycache_bias + u);
                us[5] = __ldg(s.cu + u);
                us[6] = hud ? __ldg(s.cut + rc1.ud) : 0.0f;
            }
        };
        // Producer warp pw: round r's pe rows pw, pw + 8, pw + 16, pw + 24 and
        // their scalars, then (pw < 6) a Gram tile and the entries of the
        // round's system M that it holds, or (pw == 6) the per-rating weights.
        auto produce = [&](uint32_t r) {
            const int pw = warp - kCW;
            float* dst = buf + (size_t)(r & 1) * kRound * stride;
            float* Mb = mbuf + (size_t)(r & 1) * kRound * kMS;
            float* V = vec + (size_t)(r & 1) * kVecs * kRound;
            const uint32_t m = round_len(r);
            const bool valid = lane < (int)m;
            const Rec mine = rc1;
            if ((lane & (kPW - 1)) == pw) {
                // bu_t, cu_t as user_scalars forms them (src/tsvdx4p.rs:690-708)
                const float bu = valid ? us[0] + us[1] + us[2] * mine.dev + us[3] + us[4] : 0.0f;
                const float cu = valid ? us[5] + us[6] : 0.0f;
                float* row = dst + (size_t)lane * stride;
                row[Fs] = bu;
                row[Fs + 1] = cu;
                row[Fs + 2] = mine.res;
                row[Fs + 3] = __uint_as_float(mine.key);
            }
            // ratings pw + 16 and pw + 24: their user rows are loaded now, while
            // ratings pw and pw + 8 (loaded a phase earlier) are staged; rows
            // m..31 of a partial round are zero
            {
                const uint32_t j2 = pw + 16, j3 = pw + 24;
                const uint32_t u2 = rec_id(__shfl_sync(kFull, mine.key, j2));
                const uint32_t u3 = rec_id(__shfl_sync(kFull, mine.key, j3));
                float x2[VPL], y2[VPL], x3[VPL], y3[VPL];
#pragma unroll
                for (int v = 0; v < VPL; ++v) x2[v] = y2[v] = x3[v] = y3[v] = 0.0f;
                if (j2 < m) pe_rows<VPL, BF>(s, bf, u2, lane, x2, y2);
                if (j3 < m) pe_rows<VPL, BF>(s, bf, u3, lane, x3, y3);
                const uint32_t j0 = pw, j1 = pw + kPW;
                const float d0 = __shfl_sync(kFull, mine.dev, j0), d1 = __shfl_sync(kFull, mine.dev, j1);
                const float d2 = __shfl_sync(kFull, mine.dev, j2), d3 = __shfl_sync(kFull, mine.dev, j3);
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    px0[v] = px0[v] + d0 * py0[v];
                    px1[v] = px1[v] + d1 * py1[v];
                }
                stage_row<VPL>(dst + (size_t)j0 * stride, hl + (size_t)j0 * hp, hl + (size_t)(kRound + j0) * hp, lane, px0);
                stage_row<VPL>(dst + (size_t)j1 * stride, hl + (size_t)j1 * hp, hl + (size_t)(kRound + j1) * hp, lane, px1);
#pragma unroll
                for (int v = 0; v < VPL; ++v) {
                    x2[v] = x2[v] + d2 * y2[v];
                    x3[v] = x3[v] + d3 * y3[v];
                }
                stage_row<VPL>(dst + (size_t)j2 * stride, hl + (size_t)j2 * hp, hl + (size_t)(kRound + j2) * hp, lane, x2);
                stage_row<VPL>(dst + (size_t)j3 * stride, hl + (size_t)j3 * hp, hl + (size_t)(kRound + j3) * hp, lane, x3);
            }
            // all rows of the round are in place before the Gram products
            asm volatile("bar.sync 2, %0;" ::"r"(kPW * 32) : "memory");
            const uint32_t fbl = rec_fbin(mine.key);
            // the round's ratings of each frequency bin (valid ratings only)
            const unsigned same = __match_any_sync(kFull, valid ? fbl : 64u + (uint32_t)lane);
            if (pw < 6) {
                // G = PE PE^T on the tensor cores, from BF16 high and low
                // parts of pe (three products: error ~2^-16 of |pe_i||pe_j|).
                // Tile pw of the six 16x8 tiles (rows x columns) that hold
                // every pair row < column.
                const int mt = pw < 4 ? 0 : 1, nt = pw < 4 ? pw : pw - 2;
                const int gid = lane >> 2, tig = lane & 3;
                // ldmatrix row addresses: A (16x16) as four 8x8 matrices
                // (rows 0-7 | 8-15) x (k 0-7 | 8-15); B's high and low parts
                // (8 pe rows x k 0-7 | 8-15) in one x4
                const uint32_t hl_s = smem_u32(hl);
                const int ar = mt * 16 + (lane & 7) + 8 * ((lane >> 3) & 1), ak = 8 * (lane >> 4);
                const uint32_t a_hi = hl_s + (uint32_t)(ar * hp + 2 * ak);
                const uint32_t a_lo = a_hi + (uint32_t)(kRound * hp);
                const int br = nt * 8 + (lane & 7), bk = 8 * ((lane >> 3) & 1);
                const uint32_t b_hl = hl_s + (uint32_t)(((lane >> 4) * kRound + br) * hp + 2 * bk);
                float d[6][4] = {};
#pragma unroll 2
                for (uint32_t k0 = 0; k0 < Fs; k0 += 32) {
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        const uint32_t kb = 2 * (k0 + 16 * hh);
                        uint32_t ah[4], al[4], bb[4];
                        ldmatrix_x4(ah, a_hi + kb);
                        ldmatrix_x4(al, a_lo + kb);
                        ldmatrix_x4(bb, b_hl + kb);
                        const uint32_t bh[2] = {bb[0], bb[1]}, bl[2] = {bb[2], bb[3]};
                        mma_bf16(d[3 * hh], al, bh);
                        mma_bf16(d[3 * hh + 1], ah, bl);
                        mma_bf16(d[3 * hh + 2], ah, bh);
                    }
                }
                // The round's errors solve err = C - M err with M unit lower
                // triangular: M_ji (i < j) is the effect of err_i on rating j
                // through q (a_i^(j-1-i) G_ij), the q^f row of a shared bin
                // (a_f^(same-bin ratings between) G_ij) and the item biases.
                // This lane's four entries (i, j) give M_ji and M_ij = 0.
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float g = ((d[0][e] + d[1][e]) + (d[3][e] + d[4][e])) + (d[2][e] + d[5][e]);
                    const int ii = mt * 16 + gid + 8 * (e >> 1), jj = nt * 8 + 2 * tig + (e & 1);
                    const uint32_t ki = __shfl_sync(kFull, mine.key, ii), kj = __shfl_sync(kFull, mine.key, jj);
                    const unsigned samej = __shfl_sync(kFull, same, jj);
                    if (ii < jj) {
                        float v = 0.0f;
                        if (jj < (int)m) {
                            const float cui = dst[(size_t)ii * stride + Fs + 1], cuj = dst[(size_t)jj * stride + Fs + 1];
                            const bool same_f = rec_fbin(ki) == rec_fbin(kj), same_t = rec_tbin(ki) == rec_tbin(kj);
                            const float bias_lr = p.lr_ib + (same_t ? p.lr_ti : 0.0f) + (same_f ? p.lr_ibf : 0.0f);
                            const unsigned between = ((1u << jj) - 1u) & ~((2u << ii) - 1u);
                            v = cuj * cui * bias_lr + p.lr_i * apow[jj - 1 - ii] * g +
                                (same_f ? p.lr_iqf * fpow[__popc(samej & between)] * g : 0.0f);
                        }
                        Mb[(size_t)jj * kMS + ii] = v;
                        Mb[(size_t)ii * kMS + jj] = 0.0f;
                    } else if (ii == jj) {
                        Mb[(size_t)ii * kMS + ii] = 0.0f;
                    }
                }
            } else if (pw == 6) {
                // per-rating weights of the round (j = lane)
                const unsigned below = (1u << lane) - 1u, above = ~((2u << lane) - 1u);
                const unsigned earlier = same & below;
                V[lane] = apow[lane];                                       // a_i^j
                V[kRound + lane] = fpow[__popc(earlier)];                   // a_f^(earlier ratings of the bin)
                V[2 * kRound + lane] = valid ? apow[valid ? m - 1 - lane : 0] : 0.0f;  // a_i^(m-1-j)
                V[3 * kRound + lane] = fpow[__popc(same & above)];          // a_f^(later ratings of the bin)
                // the first rating of a bin applies the decay of all its ratings to the bin's row
                V[4 * kRound + lane] = (valid && earlier == 0u) ? fpow[__popc(same)] : 1.0f;
                V[5 * kRound + lane] = __uint_as_float(fbl);
                if (lane == 0) V[6 * kRound] = apow[m];                     // a_i^m
                // the previous rating of the same bin in the round, or -1
                V[7 * kRound + lane] = __int_as_float(earlier ? 31 - __clz((int)earlier) : -1);
                V[8 * kRound + lane] = __uint_as_float(rec_tbin(mine.key));
            }
            // the next rounds' loads
            rc1 = rc2;
            if (r + 1 < rounds) {
                fetch_scalars(r + 1);
                fetch_rows0(r + 1);
            }
            fetch_records(r + 2, rc2);
        };
        if (warp >= kCW) {
            fetch_records(0, rc1);
            fetch_records(1, rc2);
            fetch_scalars(0);
            fetch_rows0(0);
            produce(0);
        }
        __syncthreads();
        for (uint32_t r = 0; r < rounds; ++r) {
            if (warp >= kCW) {
                if (r + 1 < rounds) produce(r + 1);
            } else {
                // Lookahead over the round's m ratings (all of one item): with
                // q_k, qf_k the item rows before rating k, and pe_k fixed in
                // the item stratum,
                //   q_k . pe_k = a_i^k (q_0 . pe_k) - lr_i sum_{j<k} a_i^(k-1-j) err_j G_jk
                // and likewise for the q^f row of pe_k's frequency bin over the
                // earlier ratings of the same bin. The dots with q_0 are taken
                // once per round; the round's updates are applied in closed form,
                //   q_m = a_i^m q_0 - lr_i sum_k a_i^(m-1-k) err_k pe_k.
                const float* src = buf + (size_t)(r & 1) * kRound * stride;
                const float* Mb = mbuf + (size_t)(r & 1) * kRound * kMS;
                const float* V = vec + (size_t)(r & 1) * kVecs * kRound;
                const uint32_t m = round_len(r);
                const float* myrow = src + (size_t)lane * stride;
                const uint32_t keyl = __float_as_uint(myrow[Fs + 3]);
                const uint32_t fbl = rec_fbin(keyl);
                // partial dots of pe_lane with q_0 and q^f_0[fb] over this warp's stripes
#pragma unroll
                for (int t = 0; t < CPL; ++t) {
                    const uint32_t sc = warp + kCW * t;
                    if (sc < NS) qsh[32 * sc + lane] = qv[t];
                }
                __syncwarp();
                {
                    float s0 = 0.0f, s1 = 0.0f, e0 = 0.0f, e1 = 0.0f;
#pragma unroll
                    for (int t = 0; t < CPL; ++t) {
                        const uint32_t sc = warp + kCW * t;
                        if (sc < NS) {
                            const float4* x4 = reinterpret_cast<const float4*>(myrow + 32 * sc);
                            const float4* y4 = reinterpret_cast<const float4*>(qsh + 32 * sc);
                            const float4* z4 = reinterpret_cast<const float4*>(qfs + (size_t)fbl * qs + 32 * sc);
#pragma unroll
                            for (int k4 = 0; k4 < 8; ++k4) {
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
                        }
                    }
                    pd[(2 * warp) * kRound + lane] = s0 + s1;
                    pd[(2 * warp + 1) * kRound + lane] = e0 + e1;
                }
                asm volatile("bar.sync 1, %0;" ::"r"(kCW * 32) : "memory");
                float wb = 0.0f;
                if (warp == 0) {
                    const float sq = (pd[lane] + pd[2 * kRound + lane]) + (pd[4 * kRound + lane] + pd[6 * kRound + lane]);
                    const float sf =
                        (pd[kRound + lane] + pd[3 * kRound + lane]) + (pd[5 * kRound + lane] + pd[7 * kRound + lane]);
                    const float bu_t = myrow[Fs], cu_t = myrow[Fs + 1], res = myrow[Fs + 2];
                    const uint32_t tb = rec_tbin(keyl);
                    const bool valid = lane < (int)m;
                    const float bi0 = sst[0] + sst[1 + tb] + sst[65 + fbl];
                    float x = ((gb + bu_t + bi0 * cu_t) + (V[lane] * sq + V[kRound + lane] * sf)) - res;
                    x = valid ? x : 0.0f;
                    // Forward substitution in blocks of four: each block's
                    // four values are broadcast at once, every lane solves
                    // the block's 4x4 system, and the lanes past the block
                    // subtract its contributions. M is zero on and above the
                    // diagonal, so the lanes of the block get their own value
                    // and earlier lanes keep theirs.
                    const float* Mr = Mb + (size_t)lane * kMS;
#pragma unroll
                    for (int c = 0; c < kRound; c += 4) {
                        const float s0 = __shfl_sync(kFull, x, c), s1 = __shfl_sync(kFull, x, c + 1);
                        const float s2 = __shfl_sync(kFull, x, c + 2), s3 = __shfl_sync(kFull, x, c + 3);
                        const float* B1 = Mb + (size_t)(c + 1) * kMS + c;
                        const float* B2 = Mb + (size_t)(c + 2) * kMS + c;
                        const float* B3 = Mb + (size_t)(c + 3) * kMS + c;
                        const float e1 = fmaf(-B1[0], s0, s1);
                        const float e2 = fmaf(-B2[1], e1, fmaf(-B2[0], s0, s2));
                        const float e3 = fmaf(-B3[2], e2, fmaf(-B3[1], e1, fmaf(-B3[0], s0, s3)));
                        x = fmaf(-Mr[c + 3], e3, fmaf(-Mr[c + 2], e2, fmaf(-Mr[c + 1], e1, fmaf(-Mr[c], s0, x))));
                    }
                    const float wq = valid ? p.lr_i * V[2 * kRound + lane] * x : 0.0f;
                    const float wf = valid ? p.lr_iqf * V[3 * kRound + lane] * x : 0.0f;
                    const int pv = __float_as_int(V[7 * kRound + lane]);
                    ap[lane] = make_float4(wq, wf, V[4 * kRound + lane], __uint_as_float(fbl | (uint32_t)(pv + 1) << 8));
                    wb = valid ? x * cu_t : 0.0f;
                    sv[2 * kRound + lane] = wb;
                }
                asm volatile("bar.sync 1, %0;" ::"r"(kCW * 32) : "memory");
                // q and q^f stripes, kChunk ratings at a time: the chunk's pe
                // and q^f values are loaded together, a rating whose bin an
                // earlier rating of the chunk updated takes that value from
                // registers, and the chunk's rows are stored at its end.
                if (warp >= 2) {
                    // item biases, beside the q and q^f updates of warps 0
                    // and 1 (at f <= 64 warps 2 and 3 hold no stripes): warp 2
                    // the item bias and the time-bin biases, warp 3 the
                    // frequency-bin biases
                    if (warp == 2) {
                        const float sw = warp_sum(sv[2 * kRound + lane]);
                        if (lane == 0) sst[0] = sst[0] - p.lr_ib * sw;
                    }
                    const int vo = warp == 2 ? 8 : 5;  // the ratings' bins: tb (vector 8) or fb (vector 5)
                    float d0 = 0.0f, d1 = 0.0f;
#pragma unroll 8
                    for (int c = 0; c < kRound; ++c) {
                        const float e = sv[2 * kRound + c];
                        const uint32_t bk = __float_as_uint(V[vo * kRound + c]);
                        d0 += lane == (int)bk ? e : 0.0f;
                        d1 += lane + 32 == (int)bk ? e : 0.0f;
                    }
                    const float lr = warp == 2 ? p.lr_ti : p.lr_ibf;
                    float* bb = sst + (warp == 2 ? 1 : 65);
                    bb[lane] = bb[lane] - lr * d0;
                    bb[lane + 32] = bb[lane + 32] - lr * d1;
                }
                const float am = V[6 * kRound];
#pragma unroll
                for (int t = 0; t < CPL; ++t) qv[t] *= am;
#pragma unroll 1
                for (int c0 = 0; c0 < kRound; c0 += kChunk) {
                    float pk[kChunk][CPL], ol[kChunk][CPL], nv[kChunk][CPL];
                    float4 w4[kChunk];
#pragma unroll
                    for (int u = 0; u < kChunk; ++u) {
                        w4[u] = ap[c0 + u];
                        const uint32_t fk = __float_as_uint(w4[u].w) & 0xffu;
#pragma unroll
                        for (int t = 0; t < CPL; ++t) {
                            const uint32_t sc = warp + kCW * t;
                            pk[u][t] = sc < NS ? src[(size_t)(c0 + u) * stride + 32 * sc + lane] : 0.0f;
                            ol[u][t] = sc < NS ? qfs[(size_t)fk * qs + 32 * sc + lane] : 0.0f;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kChunk; ++u) {
                        const float wq = w4[u].x, wf = w4[u].y, dk = w4[u].z;
                        const int pv = (int)(__float_as_uint(w4[u].w) >> 8) - 1;
#pragma unroll
                        for (int t = 0; t < CPL; ++t) {
                            qv[t] = fmaf(-wq, pk[u][t], qv[t]);
                            float o = ol[u][t];
#pragma unroll
                            for (int u2 = 0; u2 < u; ++u2) o = pv == c0 + u2 ? nv[u2][t] : o;
                            nv[u][t] = fmaf(-wf, pk[u][t], dk * o);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kChunk; ++u) {
                        // (ratings m..31 of a partial round would store stale rows)
                        if (c0 + u >= (int)m) break;
                        const uint32_t fk = __float_as_uint(w4[u].w) & 0xffu;
#pragma unroll
                        for (int t = 0; t < CPL; ++t) {
                            const uint32_t sc = warp + kCW * t;
                            if (sc < NS) qfs[(size_t)fk * qs + 32 * sc + lane] = nv[u][t];
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (warp < kCW) {
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const uint32_t sc = warp + kCW * t;
                if (sc < NS) s.ifeat[(size_t)i * Fs + 32 * sc + lane] = qv[t];
            }
        }
        if (threadIdx.x < 64) {
            const uint32_t t = threadIdx.x;
            if (t == 0) s.ibias[i] = sst[0];
            if (t < T) s.bit_bin[(size_t)i * T + t] = sst[1 + t];
            if (t < NF) s.ibias_freq[(size_t)i * NF + t] = sst[65 + t];
        }
        for (uint32_t e = threadIdx.x; e < NF * Fs; e += blockDim.x)
            __stcg(s.ifeat_freq + (size_t)i * NF * Fs + e, qfs[(e / Fs) * qs + e % Fs]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// n_feat > 256 (the tsvdx4 400lm ... 4800lm jobs, tsvdx4p up to 16000): rows
// of Fs = 256 k columns. A warp's unit keeps its own rows in global memory
// (they are private to it, and each lane reads back only what it wrote) and
// takes each rating in two passes over 256-column slices: the dot product,
// then the updates. Per element the arithmetic is that of the narrow kernels.
// ---------------------------------------------------------------------------
constexpr int kWV = 8;                   // values per lane in a slice
constexpr uint32_t kSlice = 32 * kWV;    // columns per slice

__global__ void __launch_bounds__(kThreads) k_user_strat_wide(DeviceState s, EpochParams p,
                                                              const uint32_t* __restrict__ order, uint32_t n_work) {
    using R8 = Row<kWV>;
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    float th[4];
    load_thresholds(s, th);
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
        float* pu_row = s.ufeat + (size_t)u * Fs;
        float* p2_row = s.ufeat2 + (size_t)u * Fs;
        float* su_row = s.ycache + (size_t)u * Fs;
        float* sq_row = s.g_user + (size_t)u * Fs;  // the NSVD1 error sum, then the user's gradient
        float sub;
        if (p.use_ycache) {
            sub = __ldcg(s.ycache_bias + u);
        } else {
            sub = 0.0f;
            for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                float su[kWV], sb = 0.0f;
#pragma unroll
                for (int v = 0; v < kWV; ++v) su[v] = 0.0f;
                const Rec* rr = s.rec + start;
                gather_rows8<kWV>(s.yfeat + c0, c0 == 0 ? s.ybias : nullptr, Fs, end - start,
                                  [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su, sb);
                if (p.full_su) {
                    const uint32_t* pp = s.pr_item + ps;
                    gather_rows8<kWV>(s.yfeat + c0, c0 == 0 ? s.ybias : nullptr, Fs, pe - ps,
                                      [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sb);
                }
#pragma unroll
                for (int v = 0; v < kWV; ++v) su[v] = su[v] / norm;
                R8::store(su_row + c0, lane, su);
                if (c0 == 0) sub = sb / norm;
            }
            if (lane == 0) s.ycache_bias[u] = sub;
        }
        {
            const float z[kWV] = {};
            for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) R8::store(sq_row + c0, lane, z);
        }
        float ub = __ldcg(s.ubias + u), al = __ldcg(s.alpha_u + u), cuu = __ldcg(s.cu + u);
        float bb0 = lane < (int)T ? __ldcg(s.but_bin + (size_t)u * T + lane) : 0.0f;
        float bb1 = lane + 32 < (int)T ? __ldcg(s.but_bin + (size_t)u * T + 32 + lane) : 0.0f;
        float sum_err = 0.0f;
        const float gb = s.gbias;
        for (uint64_t base = start; base < end; base += 32) {
            const uint32_t cnt = (uint32_t)(end - base < 32 ? end - base : 32);
            Rec mine{};
            if (lane < (int)cnt) mine = load_rec(s.rec + base + lane);
            for (uint32_t j = 0; j < cnt; ++j) {
                const Rec r = shfl_rec(mine, j);
                const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
                const bool hud = r.ud < s.n_ud;
                const float* qe_row = s.qe0 + (size_t)i * Fs;  // q_i + q^f_{i,0} (low_memory: bin 0)
                const float ib = __ldg(s.ibias + i);
                const float bit = __ldg(s.bit_bin + (size_t)i * T + tb);
                const float ibf = __ldg(s.ibias_freq + (size_t)i * NF);
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
                for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                    float qe[kWV], pu[kWV], su[kWV], p2[kWV];
                    R8::load_nc(qe_row + c0, lane, qe);
                    R8::load_cg(pu_row + c0, lane, pu);
                    R8::load_cg(su_row + c0, lane, su);
                    R8::load_cg(p2_row + c0, lane, p2);
#pragma unroll
                    for (int v = 0; v < kWV; ++v) part += qe[v] * ((pu[v] + su[v]) + dv * p2[v]);
                }
                const float dot = warp_sum(part);
                const float err = rating_err(s, th, gb + bu_t + bi_t * cu_t + dot, r.res);
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
                for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                    float qev[kWV], pu[kWV], p2[kWV], sq[kWV];
                    R8::load_nc(qe_row + c0, lane, qev);
                    R8::load_cg(pu_row + c0, lane, pu);
                    R8::load_cg(p2_row + c0, lane, p2);
                    R8::load_cg(sq_row + c0, lane, sq);
#pragma unroll
                    for (int v = 0; v < kWV; ++v) {
                        const float qe = qev[v];
                        const float pk = pu[v], p2k = p2[v];
                        sq[v] += err * qe;
                        pu[v] = pk - p.lr_u * (err * qe + p.reg_u * pk);
                        p2[v] = p2k - p.lr_u2 * (err * qe * dv + p.reg_u2 * p2k);
                    }
                    R8::store(pu_row + c0, lane, pu);
                    R8::store(p2_row + c0, lane, p2);
                    R8::store(sq_row + c0, lane, sq);
                }
            }
        }
        if (lane == 0) {
            s.ubias[u] = ub;
            s.alpha_u[u] = al;
            s.cu[u] = cuu;
        }
        if (lane < (int)T) s.but_bin[(size_t)u * T + lane] = bb0;
        if (lane + 32 < (int)T) s.but_bin[(size_t)u * T + 32 + lane] = bb1;
        for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
            float g[kWV];
            R8::load_cg(sq_row + c0, lane, g);
#pragma unroll
            for (int v = 0; v < kWV; ++v) g[v] = g[v] / norm;
            R8::store(sq_row + c0, lane, g);
        }
        if (lane == 0) s.e_user[u] = sum_err / norm;
    }
}

// Item stratum for wide rows: one warp per item, the item's q and q^f rows in
// global memory, every item on the one-warp chain.
__global__ void __launch_bounds__(kThreads) k_item_wide(DeviceState s, EpochParams p) {
    using R8 = Row<kWV>;
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, NF = s.NF;
    float th[4];
    load_thresholds(s, th);
    const float gb = s.gbias;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&s.counters[2], 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= s.n_item_work) break;
        const uint32_t i = s.item_work[k];
        const uint64_t a = s.item_off[i], b = s.item_off[i + 1];
        if (a == b) continue;
        float* q_row = s.ifeat + (size_t)i * Fs;
        float* qf_base = s.ifeat_freq + (size_t)i * NF * Fs;
        ItemState st = load_item_state(s, i, lane);
        for (uint64_t base = a; base < b; base += 32) {
            const uint32_t cnt = (uint32_t)(b - base < 32 ? b - base : 32);
            Rec mine{};
            float bu_l = 0.0f, cu_l = 0.0f;
            if (lane < (int)cnt) {
                mine = load_rec(s.irec + base + lane);
                user_scalars(s, mine, bu_l, cu_l);
            }
            for (uint32_t j = 0; j < cnt; ++j) {
                const Rec r = shfl_rec(mine, j);
                const uint32_t u = rec_id(r.key), tb = rec_tbin(r.key), fb = rec_fbin(r.key);
                const float bu_t = __shfl_sync(kFull, bu_l, j), cu_t = __shfl_sync(kFull, cu_l, j);
                const float* pyc_row = s.pyc + (size_t)u * Fs;
                const float* p2_row = s.ufeat2 + (size_t)u * Fs;
                float* qf_row = qf_base + (size_t)fb * Fs;
                const float bit = __shfl_sync(kFull, tb < 32 ? st.bt0 : st.bt1, tb & 31);
                const float ibf = __shfl_sync(kFull, fb < 32 ? st.bf0 : st.bf1, fb & 31);
                const float bi_t = st.ib + bit + ibf;
                float part = 0.0f;
                for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                    float x[kWV], y[kWV], q[kWV], qf[kWV];
                    R8::load_nc(pyc_row + c0, lane, x);
                    R8::load_nc(p2_row + c0, lane, y);
                    R8::load_cg(q_row + c0, lane, q);
                    R8::load_cg(qf_row + c0, lane, qf);
#pragma unroll
                    for (int v = 0; v < kWV; ++v) part += (x[v] + r.dev * y[v]) * (q[v] + qf[v]);
                }
                const float dot = warp_sum(part);
                const float err = rating_err(s, th, gb + bu_t + bi_t * cu_t + dot, r.res);
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
                for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                    float x[kWV], y[kWV], q[kWV], qf[kWV];
                    R8::load_nc(pyc_row + c0, lane, x);
                    R8::load_nc(p2_row + c0, lane, y);
                    R8::load_cg(q_row + c0, lane, q);
                    R8::load_cg(qf_row + c0, lane, qf);
#pragma unroll
                    for (int v = 0; v < kWV; ++v) {
                        const float pev = x[v] + r.dev * y[v];
                        const float qi = q[v];
                        q[v] = qi - p.lr_i * (err * pev + p.reg_i * qi);
                        qf[v] = qf[v] - p.lr_iqf * (err * pev + p.reg_iqf * qf[v]);
                    }
                    R8::store(q_row + c0, lane, q);
                    R8::store(qf_row + c0, lane, qf);
                }
            }
        }
        store_item_state(s, i, lane, st);
    }
}

void strat_launch_wide(tsvd_model* m, const EpochParams& p) {
    const DeviceState& s = m->d;
    make_qe0(m);
    {
        ProfScope ps(m, "user_pass_stratified");
        unsigned g = persistent_grid(k_user_strat_wide, 0);
        k_user_strat_wide<<<g, kThreads, 0, m->stream>>>(s, p, s.user_work, s.n_users);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    {
        ProfScope ps(m, "y_apply");
        y_partial_passes<kWV>(m, s, 0, s.n_users);
        k_y_combine<kWV><<<ceil_div(s.n_items, kWarps), kThreads, 0, m->stream>>>(s, p);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    launch_rebuild_ycache(m, s.pyc);
    {
        ProfScope ps(m, "item_pass");
        unsigned g = persistent_grid(k_item_wide, 0);
        k_item_wide<<<g, kThreads, 0, m->stream>>>(s, p);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
}

// Whether the user stratum of the whole user set is bound by its total work
// rather than by its longest user chains: the ratings per warp at three blocks
// per SM at least the most active user's count (1.66x at the full Netflix
// shape, 0.41x on 120,000 users).
bool user_stratum_work_bound(tsvd_model* m) {
    if (m->h_max_user_cnt == 0)
        for (uint32_t c : m->h_user_cnt) m->h_max_user_cnt = std::max(m->h_max_user_cnt, c);
    int dev = 0, sms = 0;
    TSVD_CUDA(cudaGetDevice(&dev));
    TSVD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const double warps = (double)sms * 3 * kWarps;
    return (double)m->d.n_train / warps >= (double)std::max<uint32_t>(m->h_max_user_cnt, 1u);
}

void make_qe0(tsvd_model* m) {
    const DeviceState& s = m->d;
    if (!s.qe0) return;
    const unsigned grid = (unsigned)std::min<uint64_t>(((uint64_t)s.n_items * s.Fs + 255) / 256, 148ull * 32);
    k_make_qe0<<<grid, 256, 0, m->stream>>>(s.ifeat, s.ifeat_freq, s.n_items, s.Fs, s.NF, s.qe0);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

void to_bf16(tsvd_model* m, const float* src, uint64_t rows, uint64_t src_stride, void* dst) {
    const uint32_t Fs = m->d.Fs;
    const unsigned grid = (unsigned)std::min<uint64_t>((rows * Fs + 255) / 256, 148ull * 32);
    k_to_bf16<<<grid, 256, 0, m->stream>>>(src, rows, Fs, src_stride, (__nv_bfloat16*)dst);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

// One stratified epoch (Tsvdx4pModel::fit_epoch, src/tsvdx4p.rs:815-822):
// user stratum, NSVD1 delta sums and apply, ycache (and ycache_day) rebuild,
// item stratum. The item stratum's whole-block path solves a round's errors
// as a linear system, which holds for err = score - r only: with the ordinal
// head, and with the per-day terms (which that path does not stage), every
// item takes the one-warp chain.
template <int VPL, bool BF, bool BFU, bool DAY>
void strat_launch(tsvd_model* m, const EpochParams& p, const Bf16Copies& bf) {
    DeviceState s = m->d;
    if (DAY || s.raw) s.heavy_min = 0xffffffffu;
    if (DAY) TSVD_CUDA(cudaMemsetAsync(s.dyd_fix, 0, (size_t)s.n_items * s.Fs * 8, m->stream));
    if (!BF && !DAY) make_qe0(m);
    {
        ProfScope ps(m, "user_pass_stratified");
        if (!DAY && user_stratum_work_bound(m)) {
            unsigned g = persistent_grid(k_user_strat<VPL, BF, DAY, 3>, 0);
            k_user_strat<VPL, BF, DAY, 3><<<g, kThreads, 0, m->stream>>>(s, p, bf, s.user_work, s.n_users);
        } else {
            unsigned g = persistent_grid(k_user_strat<VPL, BF, DAY>, 0);
            k_user_strat<VPL, BF, DAY><<<g, kThreads, 0, m->stream>>>(s, p, bf, s.user_work, s.n_users);
        }
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    {
        ProfScope ps(m, "y_apply");
        y_partial_passes<VPL>(m, s, 0, s.n_users);
        k_y_combine<VPL><<<ceil_div(s.n_items, kWarps), kThreads, 0, m->stream>>>(s, p);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    if (BF) to_bf16(m, s.yfeat, s.n_items, s.Fs, m->m_bf_yfeat.p);
    launch_rebuild_ycache(m, s.pyc);
    if (DAY) rebuild_ycache_day(m);
    if (BFU) {
        ProfScope ps(m, "bf16_copies");
        to_bf16(m, s.pyc, s.n_users, s.Fs, m->m_bf_pyc.p);
        to_bf16(m, s.ufeat2, s.n_users, s.Fs, m->m_bf_ufeat2.p);
    }
    {
        ProfScope ps(m, "item_pass");
        const size_t smem = (size_t)item_smem(s.Fs, s.NF).total * sizeof(float);
        auto kern = k_item_pass<VPL, BFU, DAY>;
        TSVD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int dev = 0, sms = 0, per_sm = 0;
        TSVD_CUDA(cudaGetDevice(&dev));
        TSVD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        TSVD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kItemThreads, smem));
        const unsigned g = (unsigned)(sms * std::max(per_sm, 1));
        kern<<<g, kItemThreads, smem, m->stream>>>(s, p, bf);
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

// (With the per-day terms the fold-in's yfeat_day deltas land in dyd_fix,
// which the next stratified epoch clears before its user stratum.)
template <int VPL>
void foldin_launch(tsvd_model* m, const EpochParams& p, const uint32_t* d_users, uint32_t n) {
    make_qe0(m);
    if (m->d.dyd_fix) {
        unsigned g = persistent_grid(k_user_strat<VPL, false, true>, 0);
        k_user_strat<VPL, false, true><<<g, kThreads, 0, m->stream>>>(m->d, p, Bf16Copies{}, d_users, n);
    } else {
        unsigned g = persistent_grid(k_user_strat<VPL, false, false>, 0);
        k_user_strat<VPL, false, false><<<g, kThreads, 0, m->stream>>>(m->d, p, Bf16Copies{}, d_users, n);
    }
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

// ---------------------------------------------------------------------------
// A sharded run's steps (one process per GPU, users and items in contiguous
// blocks): the user stratum of a user block with the block's NSVD1 delta sums,
// the apply of the summed deltas with the cache rebuild, and the item stratum
// of an item block. The exchanges between them are the caller's collectives.
// ---------------------------------------------------------------------------
template <int VPL, bool DAY>
void shard_user_launch(tsvd_model* m, const EpochParams& p, const uint32_t* work, uint32_t n, uint32_t u_lo,
                       uint32_t u_hi, float* sums, float* sums_e) {
    const DeviceState& s = m->d;
    if (!DAY) make_qe0(m);
    {
        ProfScope ps(m, "user_pass_stratified");
        if (s.Fs > kSlice) {
            unsigned g = persistent_grid(k_user_strat_wide, 0);
            k_user_strat_wide<<<g, kThreads, 0, m->stream>>>(s, p, work, n);
        } else {
            unsigned g = persistent_grid(k_user_strat<VPL, false, DAY>, 0);
            k_user_strat<VPL, false, DAY><<<g, kThreads, 0, m->stream>>>(s, p, Bf16Copies{}, work, n);
        }
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    }
    ProfScope ps(m, "y_apply");
    y_partial_passes<VPL>(m, s, u_lo, u_hi);
    k_y_block_sums<VPL><<<ceil_div(s.n_items, kWarps), kThreads, 0, m->stream>>>(s, sums, sums_e);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL, bool DAY>
void shard_item_launch(tsvd_model* m, const EpochParams& p, const uint32_t* work, uint32_t n) {
    DeviceState s = m->d;
    s.item_work = work;
    s.n_item_work = n;
    if (DAY || s.raw) s.heavy_min = 0xffffffffu;
    ProfScope ps(m, "item_pass");
    if (s.Fs > kSlice) {
        unsigned g = persistent_grid(k_item_wide, 0);
        k_item_wide<<<g, kThreads, 0, m->stream>>>(s, p);
    } else {
        const size_t smem = (size_t)item_smem(s.Fs, s.NF).total * sizeof(float);
        auto kern = k_item_pass<VPL, false, DAY>;
        TSVD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int dev = 0, sms = 0, per_sm = 0;
        TSVD_CUDA(cudaGetDevice(&dev));
        TSVD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        TSVD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kItemThreads, smem));
        kern<<<(unsigned)(sms * std::max(per_sm, 1)), kItemThreads, smem, m->stream>>>(s, p, Bf16Copies{});
    }
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

// Units lo..hi-1 of a count table, heaviest first (ties by id).
std::vector<uint32_t> block_work(uint32_t lo, uint32_t hi, const std::function<uint64_t(uint32_t)>& count) {
    std::vector<uint32_t> w(hi - lo);
    std::iota(w.begin(), w.end(), lo);
    std::stable_sort(w.begin(), w.end(), [&](uint32_t a, uint32_t b) { return count(a) > count(b); });
    return w;
}

void upload_work(tsvd_model* m, const std::vector<uint32_t>& w) {
    if (m->m_shard_work.bytes < std::max<size_t>(w.size(), 1) * 4) m->m_shard_work.alloc(std::max<size_t>(w.size(), 1) * 4);
    if (!w.empty())
        TSVD_CUDA(cudaMemcpyAsync(m->m_shard_work.p, w.data(), w.size() * 4, cudaMemcpyHostToDevice, m->stream));
    TSVD_CUDA(cudaStreamSynchronize(m->stream));  // `w` leaves scope
}

void check_shardable(const tsvd_model* m) {
    if (m->opts.schedule != TSVD_SCHED_STRATIFIED || m->opts.precision != TSVD_PREC_FP32)
        throw Error(TSVD_ERR_UNSUPPORTED, "a sharded run needs the stratified schedule with FP32 reads");
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
        bf.pyc = m->m_bf_pyc.as<__nv_bfloat16>();
        bf.ufeat2 = m->m_bf_ufeat2.as<__nv_bfloat16>();
    }
    const int vpl = (int)(s.Fs / 32);
    if (s.Fs > kSlice) {  // n_feat > 256: low_memory, FP32
        strat_launch_wide(m, p);
    } else if (s.dyd_fix) {  // low_memory = false (FP32 only)
        TSVD_DISPATCH(vpl, (strat_launch<V, false, false, true>(m, p, bf)));
    } else if (prec == TSVD_PREC_FP32) {
        TSVD_DISPATCH(vpl, (strat_launch<V, false, false, false>(m, p, bf)));
    } else if (prec == TSVD_PREC_BF16_READ) {
        TSVD_DISPATCH(vpl, (strat_launch<V, true, false, false>(m, p, bf)));
    } else {
        TSVD_DISPATCH(vpl, (strat_launch<V, true, true, false>(m, p, bf)));
    }
}

}  // namespace tsvd

// ---------------------------------------------------------------------------
// Fold-in and user reset entry points.
// ---------------------------------------------------------------------------
extern "C" int tsvd_foldin(tsvd_model* m, const uint32_t* users, uint64_t n, uint32_t passes) {
    using namespace tsvd;
    if (!m || (!users && n)) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (n == 0 || passes == 0) return;
        if (n >= (1ull << 32)) throw Error(TSVD_ERR_INVALID, "too many users");
        if (m->d.Fs > kSlice) throw Error(TSVD_ERR_UNSUPPORTED, "fold-in is built for n_feat up to 256");
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
    return guarded(m, [&] {
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

// ---------------------------------------------------------------------------
// Sharded-run entry points.
// ---------------------------------------------------------------------------
extern "C" int tsvd_shard_user_block(tsvd_model* m, uint64_t epoch, uint32_t u_lo, uint32_t u_hi, float* d_sums,
                                     float* d_sums_e, int64_t* d_dyd) {
    using namespace tsvd;
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        check_shardable(m);
        if (epoch == 0) throw Error(TSVD_ERR_INVALID, "epoch is 1-based");
        if (u_lo > u_hi || u_hi > m->d.n_users) throw Error(TSVD_ERR_INVALID, "user block out of range");
        if (!d_sums || !d_sums_e || (m->d.dyd_fix && !d_dyd))
            throw Error(TSVD_ERR_INVALID, "null delta buffer");
        use_device(m);
        const DeviceState& s = m->d;
        if (epoch == m->cfg.reset_u_epoch) {
            TSVD_CUDA(cudaMemsetAsync(s.ufeat, 0, m->m_ufeat.bytes, m->stream));
            TSVD_CUDA(cudaMemsetAsync(s.ufeat2, 0, m->m_ufeat2.bytes, m->stream));
        }
        TSVD_CUDA(cudaMemsetAsync(s.counters, 0, 64, m->stream));
        std::vector<uint32_t> w = block_work(u_lo, u_hi, [&](uint32_t u) { return (uint64_t)m->h_user_cnt[u]; });
        upload_work(m, w);
        EpochParams p = make_params(m);
        p.use_ycache = (m->cfg.full_su && m->ycache_valid) ? 1 : 0;
        if (s.dyd_fix) TSVD_CUDA(cudaMemsetAsync(s.dyd_fix, 0, (size_t)s.n_items * s.Fs * 8, m->stream));
        const int vpl = (int)std::min<uint32_t>(s.Fs / 32, 8);
        if (s.dyd_fix) {
            TSVD_DISPATCH(vpl, (shard_user_launch<V, true>(m, p, m->m_shard_work.as<uint32_t>(), (uint32_t)w.size(),
                                                          u_lo, u_hi, d_sums, d_sums_e)));
            TSVD_CUDA(cudaMemcpyAsync(d_dyd, s.dyd_fix, (size_t)s.n_items * s.Fs * 8, cudaMemcpyDeviceToDevice,
                                      m->stream));
        } else {
            TSVD_DISPATCH(vpl, (shard_user_launch<V, false>(m, p, m->m_shard_work.as<uint32_t>(), (uint32_t)w.size(),
                                                           u_lo, u_hi, d_sums, d_sums_e)));
        }
        m->ycache_valid = false;  // the ycache rows of the block's users were rewritten from the current y
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

extern "C" int tsvd_shard_apply(tsvd_model* m, const float* d_sums, const float* d_sums_e, const int64_t* d_dyd) {
    using namespace tsvd;
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        check_shardable(m);
        if (!d_sums || !d_sums_e || (m->d.dyd_fix && !d_dyd)) throw Error(TSVD_ERR_INVALID, "null delta buffer");
        use_device(m);
        const DeviceState& s = m->d;
        const EpochParams p = make_params(m);
        const int vpl = (int)std::min<uint32_t>(s.Fs / 32, 8);
        {
            ProfScope ps(m, "y_apply");
            TSVD_DISPATCH(vpl, (k_y_apply_sums<V><<<ceil_div(s.n_items, kWarps), kThreads, 0, m->stream>>>(
                                   s, p, d_sums, d_sums_e, s.dyd_fix ? (const long long*)d_dyd : nullptr)));
            TSVD_CUDA(cudaGetLastError());
            m->launches++;
        }
        launch_rebuild_ycache(m, s.pyc);
        rebuild_ycache_day(m);
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

extern "C" int tsvd_shard_item_block(tsvd_model* m, uint32_t i_lo, uint32_t i_hi) {
    using namespace tsvd;
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        check_shardable(m);
        if (i_lo > i_hi || i_hi > m->d.n_items) throw Error(TSVD_ERR_INVALID, "item block out of range");
        use_device(m);
        const DeviceState& s = m->d;
        if (m->h_item_off.empty()) {
            m->h_item_off.resize((size_t)s.n_items + 1);
            TSVD_CUDA(cudaMemcpy(m->h_item_off.data(), s.item_off, m->h_item_off.size() * 8, cudaMemcpyDeviceToHost));
        }
        TSVD_CUDA(cudaMemsetAsync(s.counters, 0, 64, m->stream));
        std::vector<uint32_t> w =
            block_work(i_lo, i_hi, [&](uint32_t i) { return m->h_item_off[i + 1] - m->h_item_off[i]; });
        upload_work(m, w);
        const EpochParams p = make_params(m);
        const int vpl = (int)std::min<uint32_t>(s.Fs / 32, 8);
        if (s.dyd_fix) {
            TSVD_DISPATCH(vpl, (shard_item_launch<V, true>(m, p, m->m_shard_work.as<uint32_t>(), (uint32_t)w.size())));
        } else {
            TSVD_DISPATCH(vpl, (shard_item_launch<V, false>(m, p, m->m_shard_work.as<uint32_t>(), (uint32_t)w.size())));
        }
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
        finish_epoch(m);
    });
}
