// Per-user epoch pass without software pipelining, for the two forms the
// pipelined Hogwild kernel (tsvd_epoch.cu) does not take:
//  - the per-day terms of low_memory = false (TxModel::fit_epoch,
//    src/tx.rs:846-871 su_day per run of equal dates, :1010-1036 ufeat_day
//    and the end-of-run yfeat_day update), with all users in flight
//    (Hogwild) or one after another;
//  - the sequential schedule: a single warp takes the users in get_users
//    order, so every rating sees every earlier update, which is the
//    reference's fit_epoch exactly (up to FP32 rounding of the warp-tree dot
//    products). With the ordinal head it also trains the thresholds after
//    every rating (src/tx.rs:963-972), which needs that sequential order.
// Item-side writes are atomic deltas as in the Hogwild kernel; in the
// sequential form they are plain read-modify-writes in effect.
//
// rebuild_ycache_day (src/tx.rs:420-454) is here too: one warp per (user,
// day), pr items then training items in stored order, divided by
// sqrt(count), which reproduces the reference's sums bit for bit.
#include "tsvd_epoch.cuh"

namespace tsvd {
namespace {

// OrdinalHead::grad (src/lib.rs:562-598) with the threshold gradient g_t.
__device__ __forceinline__ float ordinal_grad_t(const float (&th)[4], float score, int y, float (&gt)[4]) {
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
#pragma unroll
    for (int k = 0; k < 4; ++k) gt[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (y >= 2 && k == y - 2) gt[k] += ay1 / p_y;
        if (y <= 4 && k == y - 1) gt[k] -= ay / p_y;
    }
    return (ay - ay1) / p_y;
}

// One user, by one warp. `th` holds the ordinal thresholds (lane-uniform).
template <int VPL, bool DAY>
__device__ __forceinline__ void seq_user(const DeviceState& s, const EpochParams& p, uint32_t u, int lane,
                                         float (&th)[4]) {
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    const uint64_t start = s.user_off[u], end = s.user_off[u + 1];
    if (start == end) return;
    const uint64_t n = end - start;
    const Rec* rr = s.rec + start;
    const uint64_t ps = s.pr_off[u], pe_ = s.pr_off[u + 1];
    const uint64_t total = n + (p.full_su ? (pe_ - ps) : 0);
    const float norm = sqrtf((float)total);

    // su (src/tx.rs:800-822) from the current y
    float su[VPL], sub = 0.0f;
#pragma unroll
    for (int v = 0; v < VPL; ++v) su[v] = 0.0f;
    gather_y8<VPL>(s, n, [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su, sub);
    if (p.full_su) {
        const uint32_t* pp = s.pr_item + ps;
        gather_y8<VPL>(s, pe_ - ps, [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sub);
    }
#pragma unroll
    for (int v = 0; v < VPL; ++v) su[v] = su[v] / norm;
    sub = sub / norm;
    Row<VPL>::store(s.ycache + (size_t)u * Fs, lane, su);
    if (lane == 0) s.ycache_bias[u] = sub;

    float pu[VPL], p2[VPL], seq[VPL];
    Row<VPL>::load_cg(s.ufeat + (size_t)u * Fs, lane, pu);
    Row<VPL>::load_cg(s.ufeat2 + (size_t)u * Fs, lane, p2);
#pragma unroll
    for (int v = 0; v < VPL; ++v) seq[v] = 0.0f;
    float ub = __ldcg(s.ubias + u), al = __ldcg(s.alpha_u + u), cuu = __ldcg(s.cu + u);
    float sum_err = 0.0f;
    const float gb = s.gbias;

    // per-day state of the current run of equal dates
    float sud[VPL], seqd[VPL], pud[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) sud[v] = seqd[v] = pud[v] = 0.0f;
    float norm_day = 1.0f;
    uint64_t run0 = 0, run1 = 0;  // [run0, run1] = ratings of the run

    for (uint64_t t = 0; t < n; ++t) {
        const Rec r = load_rec(rr + t);
        const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
        // low_memory trains frequency bin 0 only (cur_freq_bin is set in the
        // per-day branch alone, src/tx.rs:834,873)
        const uint32_t f = DAY ? rec_fbin(r.key) : 0u;
        const uint32_t ud = r.ud;
        const bool hud = ud < s.n_ud;
        const float dv = r.dev;
        if (DAY && (t == 0 || t > run1)) {
            // a new run of equal dates (day_ranges, src/tx.rs:92-104)
            run0 = t;
            run1 = t;
            while (run1 + 1 < n && __ldg(&rr[run1 + 1].ud) == ud) ++run1;
#pragma unroll
            for (int v = 0; v < VPL; ++v) sud[v] = seqd[v] = 0.0f;
            float dummy = 0.0f;
            gather_rows8<VPL>(s.yfeat_day, nullptr, Fs, run1 - run0 + 1,
                              [&](uint64_t q) { return rec_id(__ldg(&rr[run0 + q].key)); }, lane, sud, dummy);
            float day_cnt = (float)(run1 - run0 + 1);
            if (p.full_su && hud) {
                const uint64_t off = s.ud_list_off[ud];
                const uint32_t pc = s.ud_pr_cnt[ud];
                gather_rows8<VPL>(s.yfeat_day, nullptr, Fs, pc,
                                  [&](uint64_t q) { return __ldg(s.ud_list_item + off + q); }, lane, sud, dummy);
                for (uint32_t k = 0; k < pc; ++k) day_cnt += 1.0f;
            }
            norm_day = sqrtf(day_cnt);
#pragma unroll
            for (int v = 0; v < VPL; ++v) sud[v] = sud[v] / norm_day;
            // su_freq is zero-filled and divided by norm_day (src/tx.rs:857,869): zero
            if (hud) Row<VPL>::load_cg(s.ufeat_day + (size_t)ud * Fs, lane, pud);
            else
#pragma unroll
                for (int v = 0; v < VPL; ++v) pud[v] = 0.0f;
        }

        // scalars: lane 0 reads (it alone writes them), then broadcasts
        float sc[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (lane == 0) {
            sc[0] = __ldcg(s.ibias + i);
            sc[1] = __ldcg(s.bit_bin + (size_t)i * T + tb);
            sc[2] = __ldcg(s.ibias_freq + (size_t)i * NF + f);
            sc[3] = hud ? __ldcg(s.cut + ud) : 0.0f;
            sc[4] = hud ? __ldcg(s.ubias_day + ud) : 0.0f;
            sc[5] = __ldcg(s.but_bin + (size_t)u * T + tb);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) sc[k] = __shfl_sync(kFull, sc[k], 0);
        const float ib = sc[0], bit = sc[1], ibf = sc[2], ct = sc[3], bud = sc[4], but = sc[5];
        const float bu_t = ub + but + al * dv + bud + sub;
        const float bi_t = ib + bit + ibf;
        const float cu_t = cuu + ct;

        float q[VPL], qf[VPL];
        Row<VPL>::load_cg(s.ifeat + (size_t)i * Fs, lane, q);
        Row<VPL>::load_cg(s.ifeat_freq + ((size_t)i * NF + f) * Fs, lane, qf);
        float part = 0.0f;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
            float pe = (pu[v] + su[v]) + dv * p2[v];
            if (DAY) {
                if (hud) pe += pud[v];
                pe += sud[v] + 0.0f;
            }
            part += pe * (q[v] + qf[v]);
        }
        const float dot = warp_sum(part);
        const float score = gb + bu_t + bi_t * cu_t + dot;
        float err = score - r.res;
        if (s.raw) {
            float gt[4];
            err = ordinal_grad_t(th, score, (int)__ldg(s.raw + start + t), gt);
            if (p.lr_t != 0.0f) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float tk = th[k];
                    th[k] -= p.lr_t * (gt[k] + p.reg_t * tk);
                }
            }
        }
        const float err_b = err * p.w_bias, err_d = err * p.w_factor;

        // bias updates (src/tx.rs:978-987)
        ub -= p.lr_ub * err_b;
        al -= p.lr_ta * err_b * dv;
        if (lane == 0) {
            s.but_bin[(size_t)u * T + tb] = but - p.lr_tu * err_b;
            if (hud) s.ubias_day[ud] = bud - p.lr_ubd * err_b;
            atomicAdd(s.ibias + i, -(p.lr_ib * (err_b * cu_t)));
            atomicAdd(s.bit_bin + (size_t)i * T + tb, -(p.lr_ti * (err_b * cu_t)));
            atomicAdd(s.ibias_freq + (size_t)i * NF + f, -(p.lr_ibf * (err_b * cu_t)));
        }
        cuu -= p.lr_cu * (err_b * bi_t + p.reg_cu * (cuu - 1.0f));

        // factor updates (src/tx.rs:992-1023)
        if (!p.sum_err_bug) sum_err += err_b;
        else
            for (uint32_t kk = 0; kk < s.F; ++kk) sum_err += err_b;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
            const float qe = q[v] + qf[v];
            const float pk = pu[v], p2k = p2[v];
            seq[v] += err_d * qe;
            if (DAY) seqd[v] += err_d * qe;
            pu[v] = pk - p.lr_u * (err_d * qe + p.reg_u * pk);
            p2[v] = p2k - p.lr_u2 * (err_d * qe * dv + p.reg_u2 * p2k);
            float pudk = 0.0f;
            if (DAY && p.has_ud && hud) {
                pudk = pud[v];
                pud[v] = pudk - p.lr_ud * (err_d * qe + p.reg_ud * pudk);
            }
            float pe = pk + dv * p2k + pudk + su[v];
            if (DAY) pe += sud[v] + 0.0f;
            q[v] = -(p.lr_i * (err_d * pe + p.reg_i * q[v]));        // delta of q_i
            qf[v] = -(p.lr_iqf * (err_d * pe + p.reg_iqf * qf[v]));  // delta of q^f_{i,f}
        }
        Row<VPL>::red_add(s.ifeat + (size_t)i * Fs, lane, q);
        Row<VPL>::red_add(s.ifeat_freq + ((size_t)i * NF + f) * Fs, lane, qf);

        if (DAY && t == run1) {
            // end of the run: ufeat_day back, NSVD1-day update of the run's
            // items (src/tx.rs:1025-1036)
            if (p.has_ud && hud) Row<VPL>::store(s.ufeat_day + (size_t)ud * Fs, lane, pud);
            for (uint64_t k = run0; k <= run1; ++k) {
                const uint32_t j = rec_id(__ldg(&rr[k].key));
                float yd[VPL];
                Row<VPL>::load_cg(s.yfeat_day + (size_t)j * Fs, lane, yd);
#pragma unroll
                for (int v = 0; v < VPL; ++v) yd[v] = -(p.lr_yd * (seqd[v] / norm_day + p.reg_yd * yd[v]));
                Row<VPL>::red_add(s.yfeat_day + (size_t)j * Fs, lane, yd);
            }
        }
        __syncwarp();  // lane 0's scalar writes before the next rating's reads
    }

    Row<VPL>::store(s.ufeat + (size_t)u * Fs, lane, pu);
    Row<VPL>::store(s.ufeat2 + (size_t)u * Fs, lane, p2);
    if (lane == 0) {
        s.ubias[u] = ub;
        s.alpha_u[u] = al;
        s.cu[u] = cuu;
    }

    // NSVD1 factor & bias updates at the end of the user (src/tx.rs:1099-1106)
    float g[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) g[v] = seq[v] / norm;
    const float eb = sum_err / norm;
    for (uint64_t base = 0; base < n; base += 32) {
        const uint32_t cnt = (uint32_t)(n - base < 32 ? n - base : 32);
        const uint32_t mine = lane < (int)cnt ? rec_id(__ldg(&rr[base + lane].key)) : 0u;
        for (uint32_t j = 0; j < cnt; j += kBatch) {
            float y[kBatch][VPL];
            uint32_t its[kBatch];
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                its[b] = __shfl_sync(kFull, mine, j + b < cnt ? j + b : cnt - 1);
                Row<VPL>::load_cg(s.yfeat + (size_t)its[b] * Fs, lane, y[b]);
            }
#pragma unroll
            for (int b = 0; b < kBatch; ++b) {
                if (j + b < cnt) {
#pragma unroll
                    for (int v = 0; v < VPL; ++v) y[b][v] = -(p.lr_y * (g[v] + p.reg_y * y[b][v]));
                    Row<VPL>::red_add(s.yfeat + (size_t)its[b] * Fs, lane, y[b]);
                    if (lane == 0) atomicAdd(s.ybias + its[b], -(p.lr_yb * eb));
                }
            }
        }
    }
    __syncwarp();
}

template <int VPL, bool DAY>
__global__ void __launch_bounds__(kThreads) k_seq_pass(DeviceState s, EpochParams p,
                                                       const uint32_t* __restrict__ order, uint32_t n_work) {
    const int lane = threadIdx.x & 31;
    float th[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (s.raw)
#pragma unroll
        for (int k = 0; k < 4; ++k) th[k] = __ldcg(s.thresholds + k);
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&s.counters[0], 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= n_work) break;
        seq_user<VPL, DAY>(s, p, order[k], lane, th);
    }
    // thresholds trained per rating exist only in the one-warp launch
    if (s.raw && p.lr_t != 0.0f && gridDim.x == 1 && threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) s.thresholds[k] = th[k];
}

// ycache_day[d] = (sum of yfeat_day over d's pr items, then its training
// items) / sqrt(count), zero for an empty list.
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_rebuild_ycache_day(DeviceState s) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * kWarps;
    for (uint64_t d = blockIdx.x * (uint64_t)kWarps + (threadIdx.x >> 5); d < s.n_ud; d += warps) {
        const uint64_t off = s.ud_list_off[d], cnt = s.ud_list_off[d + 1] - off;
        float acc[VPL], dummy = 0.0f;
#pragma unroll
        for (int v = 0; v < VPL; ++v) acc[v] = 0.0f;
        gather_rows8<VPL>(s.yfeat_day, nullptr, s.Fs, cnt, [&](uint64_t q) { return __ldg(s.ud_list_item + off + q); },
                          lane, acc, dummy);
        if (cnt > 0) {
            float c = 0.0f;
            for (uint64_t k = 0; k < cnt; ++k) c += 1.0f;
            const float nrm = sqrtf(c);
#pragma unroll
            for (int v = 0; v < VPL; ++v) acc[v] = acc[v] / nrm;
        }
        Row<VPL>::store(s.ycache_day + d * s.Fs, lane, acc);
    }
}

// The sequential pass for n_feat > 256 (low_memory, no ordinal head): one
// warp, users in get_users order; the user's rows and the rated item's rows
// are read and written in 256-column slices, in two passes per rating (the
// dot product, then the updates), with the user's NSVD1 error sum kept in the
// user's g_user row. Per element the arithmetic is seq_user's.
constexpr int kWV = 8;
constexpr uint32_t kSlice = 32 * kWV;

__global__ void __launch_bounds__(32) k_seq_wide(DeviceState s, EpochParams p, const uint32_t* __restrict__ order,
                                                 uint32_t n_work) {
    using R8 = Row<kWV>;
    const int lane = threadIdx.x & 31;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    const float gb = s.gbias;
    for (uint32_t k = 0; k < n_work; ++k) {
        const uint32_t u = order[k];
        const uint64_t start = s.user_off[u], end = s.user_off[u + 1];
        if (start == end) continue;
        const uint64_t n = end - start;
        const Rec* rr = s.rec + start;
        const uint64_t ps = s.pr_off[u], pe_ = s.pr_off[u + 1];
        const uint64_t total = n + (p.full_su ? (pe_ - ps) : 0);
        const float norm = sqrtf((float)total);
        float* pu_row = s.ufeat + (size_t)u * Fs;
        float* p2_row = s.ufeat2 + (size_t)u * Fs;
        float* su_row = s.ycache + (size_t)u * Fs;
        float* sq_row = s.g_user + (size_t)u * Fs;
        // su (src/tx.rs:800-822) from the current y, slice by slice
        float sub = 0.0f;
        for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
            float su[kWV], sb = 0.0f;
#pragma unroll
            for (int v = 0; v < kWV; ++v) su[v] = 0.0f;
            gather_rows8<kWV>(s.yfeat + c0, c0 == 0 ? s.ybias : nullptr, Fs, n,
                              [&](uint64_t q) { return rec_id(__ldg(&rr[q].key)); }, lane, su, sb);
            if (p.full_su) {
                const uint32_t* pp = s.pr_item + ps;
                gather_rows8<kWV>(s.yfeat + c0, c0 == 0 ? s.ybias : nullptr, Fs, pe_ - ps,
                                  [&](uint64_t q) { return __ldg(pp + q); }, lane, su, sb);
            }
#pragma unroll
            for (int v = 0; v < kWV; ++v) su[v] = su[v] / norm;
            R8::store(su_row + c0, lane, su);
            const float z[kWV] = {};
            R8::store(sq_row + c0, lane, z);
            if (c0 == 0) sub = sb / norm;
        }
        if (lane == 0) s.ycache_bias[u] = sub;
        float ub = __ldcg(s.ubias + u), al = __ldcg(s.alpha_u + u), cuu = __ldcg(s.cu + u);
        float sum_err = 0.0f;
        for (uint64_t t = 0; t < n; ++t) {
            const Rec r = load_rec(rr + t);
            const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
            const uint32_t ud = r.ud;
            const bool hud = ud < s.n_ud;
            const float dv = r.dev;
            float sc[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (lane == 0) {
                sc[0] = __ldcg(s.ibias + i);
                sc[1] = __ldcg(s.bit_bin + (size_t)i * T + tb);
                sc[2] = __ldcg(s.ibias_freq + (size_t)i * NF);  // low_memory trains bin 0
                sc[3] = hud ? __ldcg(s.cut + ud) : 0.0f;
                sc[4] = hud ? __ldcg(s.ubias_day + ud) : 0.0f;
                sc[5] = __ldcg(s.but_bin + (size_t)u * T + tb);
            }
#pragma unroll
            for (int c = 0; c < 6; ++c) sc[c] = __shfl_sync(kFull, sc[c], 0);
            const float ib = sc[0], bit = sc[1], ibf = sc[2], ct = sc[3], bud = sc[4], but = sc[5];
            const float bu_t = ub + but + al * dv + bud + sub;
            const float bi_t = ib + bit + ibf;
            const float cu_t = cuu + ct;
            float* q_row = s.ifeat + (size_t)i * Fs;
            float* qf_row = s.ifeat_freq + (size_t)i * NF * Fs;
            float part = 0.0f;
            for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                float q[kWV], qf[kWV], pu[kWV], su[kWV], p2[kWV];
                R8::load_cg(q_row + c0, lane, q);
                R8::load_cg(qf_row + c0, lane, qf);
                R8::load_cg(pu_row + c0, lane, pu);
                R8::load_cg(su_row + c0, lane, su);
                R8::load_cg(p2_row + c0, lane, p2);
#pragma unroll
                for (int v = 0; v < kWV; ++v) part += ((pu[v] + su[v]) + dv * p2[v]) * (q[v] + qf[v]);
            }
            const float dot = warp_sum(part);
            const float err = (gb + bu_t + bi_t * cu_t + dot) - r.res;
            const float err_b = err * p.w_bias, err_d = err * p.w_factor;
            // bias updates (src/tx.rs:978-987)
            ub -= p.lr_ub * err_b;
            al -= p.lr_ta * err_b * dv;
            if (lane == 0) {
                s.but_bin[(size_t)u * T + tb] = but - p.lr_tu * err_b;
                if (hud) s.ubias_day[ud] = bud - p.lr_ubd * err_b;
                s.ibias[i] = ib - p.lr_ib * (err_b * cu_t);
                s.bit_bin[(size_t)i * T + tb] = bit - p.lr_ti * (err_b * cu_t);
                s.ibias_freq[(size_t)i * NF] = ibf - p.lr_ibf * (err_b * cu_t);
            }
            cuu -= p.lr_cu * (err_b * bi_t + p.reg_cu * (cuu - 1.0f));
            // factor updates (src/tx.rs:992-1023)
            if (!p.sum_err_bug) sum_err += err_b;
            else
                for (uint32_t kk = 0; kk < s.F; ++kk) sum_err += err_b;
            for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                float q[kWV], qf[kWV], pu[kWV], su[kWV], p2[kWV], sq[kWV];
                R8::load_cg(q_row + c0, lane, q);
                R8::load_cg(qf_row + c0, lane, qf);
                R8::load_cg(pu_row + c0, lane, pu);
                R8::load_cg(su_row + c0, lane, su);
                R8::load_cg(p2_row + c0, lane, p2);
                R8::load_cg(sq_row + c0, lane, sq);
#pragma unroll
                for (int v = 0; v < kWV; ++v) {
                    const float qe = q[v] + qf[v];
                    const float pk = pu[v], p2k = p2[v];
                    sq[v] += err_d * qe;
                    pu[v] = pk - p.lr_u * (err_d * qe + p.reg_u * pk);
                    p2[v] = p2k - p.lr_u2 * (err_d * qe * dv + p.reg_u2 * p2k);
                    const float pe = pk + dv * p2k + 0.0f + su[v];
                    q[v] = q[v] + -(p.lr_i * (err_d * pe + p.reg_i * q[v]));
                    qf[v] = qf[v] + -(p.lr_iqf * (err_d * pe + p.reg_iqf * qf[v]));
                }
                R8::store(pu_row + c0, lane, pu);
                R8::store(p2_row + c0, lane, p2);
                R8::store(sq_row + c0, lane, sq);
                R8::store(q_row + c0, lane, q);
                R8::store(qf_row + c0, lane, qf);
            }
            __syncwarp();  // lane 0's scalar writes before the next rating's reads
        }
        if (lane == 0) {
            s.ubias[u] = ub;
            s.alpha_u[u] = al;
            s.cu[u] = cuu;
        }
        // NSVD1 factor & bias updates at the end of the user (src/tx.rs:1099-1106)
        const float eb = sum_err / norm;
        for (uint64_t t = 0; t < n; ++t) {
            const uint32_t j = rec_id(__ldg(&rr[t].key));
            for (uint32_t c0 = 0; c0 < Fs; c0 += kSlice) {
                float g[kWV], y[kWV];
                R8::load_cg(sq_row + c0, lane, g);
                R8::load_cg(s.yfeat + (size_t)j * Fs + c0, lane, y);
#pragma unroll
                for (int v = 0; v < kWV; ++v) y[v] = y[v] + -(p.lr_y * (g[v] / norm + p.reg_y * y[v]));
                R8::store(s.yfeat + (size_t)j * Fs + c0, lane, y);
            }
            if (lane == 0) s.ybias[j] = s.ybias[j] + -(p.lr_yb * eb);
            __syncwarp();
        }
    }
}

template <int VPL, bool DAY>
void launch_seq(tsvd_model* m, const EpochParams& p, const uint32_t* order, bool sequential) {
    const unsigned g = sequential ? 1u : persistent_grid(k_seq_pass<VPL, DAY>, 0);
    const unsigned threads = sequential ? 32u : (unsigned)kThreads;
    k_seq_pass<VPL, DAY><<<g, threads, 0, m->stream>>>(m->d, p, order, m->d.n_users);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL>
void launch_rebuild_day(tsvd_model* m) {
    const unsigned g = persistent_grid(k_rebuild_ycache_day<VPL>, 0);
    k_rebuild_ycache_day<VPL><<<g, kThreads, 0, m->stream>>>(m->d);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

}  // namespace

void day_epoch_pass(tsvd_model* m, const uint32_t* order, bool sequential) {
    const EpochParams p = make_params(m);
    const int vpl = (int)(m->d.Fs / 32);
    ProfScope ps(m, sequential ? "user_pass_sequential" : "user_pass_hogwild_day");
    if (m->d.Fs > kSlice) {
        // n_feat > 256: sequential only (create() rejects Hogwild there)
        if (!sequential) throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256 needs the stratified or sequential schedule");
        k_seq_wide<<<1, 32, 0, m->stream>>>(m->d, p, order, m->d.n_users);
        TSVD_CUDA(cudaGetLastError());
        m->launches++;
    } else if (m->cfg.low_memory) {
        TSVD_DISPATCH(vpl, (launch_seq<V, false>(m, p, order, sequential)));
    } else {
        TSVD_DISPATCH(vpl, (launch_seq<V, true>(m, p, order, sequential)));
    }
}

void rebuild_ycache_day(tsvd_model* m) {
    if (m->cfg.low_memory || m->d.n_ud == 0) return;
    ProfScope ps(m, "rebuild_ycache_day");
    const int vpl = (int)(m->d.Fs / 32);
    TSVD_DISPATCH(vpl, launch_rebuild_day<V>(m));
}

}  // namespace tsvd
