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
#include <algorithm>
#include <cstring>

#include "rand_stream.hpp"
#include "tsvd_epoch.cuh"

namespace tsvd {

EpochParams make_params(const tsvd_model* m) {
    const tsvd_config& c = m->cfg;
    EpochParams p;
    p.lr_u = c.lr_u; p.lr_u2 = c.lr_u2; p.lr_ub = c.lr_ub; p.lr_ubd = c.lr_ubd; p.lr_i = c.lr_i;
    p.lr_ib = c.lr_ib; p.lr_y = c.lr_y; p.lr_yb = c.lr_yb; p.lr_tu = c.lr_tu; p.lr_ti = c.lr_ti;
    p.lr_ta = c.lr_ta; p.lr_ibf = c.lr_ibf; p.lr_iqf = c.lr_iqf; p.lr_cu = c.lr_cu;
    p.reg_iqf = c.reg_iqf; p.reg_cu = c.reg_cu; p.reg_u = c.reg_u; p.reg_u2 = c.reg_u2; p.reg_i = c.reg_i;
    p.reg_y = c.reg_y;
    p.lr_ud = c.lr_ud; p.reg_ud = c.reg_ud; p.lr_yd = c.lr_yd; p.reg_yd = c.reg_yd;
    p.lr_t = c.has_ordinal_head ? c.ordinal_head.lr_t : 0.0f;
    p.reg_t = c.has_ordinal_head ? c.ordinal_head.reg_t : 0.0f;
    p.has_ud = (!c.low_memory && c.lr_ud != 0.0f) ? 1 : 0;
    p.w_bias = c.w_bias; p.w_factor = c.w_factor;
    p.nsvd_norm_exp = m->opts.nsvd_norm_exp;
    p.sum_err_bug = c.sum_err_bug;
    p.full_su = c.full_su;
    p.use_ycache = 0;
    p.stages = 4;
    return p;
}

namespace {

// ---------------------------------------------------------------------------
// Hogwild epoch, software-pipelined. The arithmetic is k_user_pass<VPL, true>'s
// (the reference's per-user pass); what changes is when data is fetched, so a
// warp stops waiting on memory between dependent ratings:
//  - the q_i and q^f_{i,0} rows of the next ST - 1 ratings are staged in a
//    per-warp shared-memory ring by cp.async, together with the item-bias
//    scalars, cut and the rating's record fields;
//  - ubias_day of the next ST - 1 ratings is prefetched into registers; when
//    one of them is on the same (user, day) as the rating just updated, the
//    prefetched value is replaced by the value just written, so every rating
//    sees the reference's sequential value;
//  - the su gather and the end-of-user y update keep 8 rows in flight.
// ---------------------------------------------------------------------------
constexpr int kStages = 4;  // default ring depth (the batched form tunes it per width)

// One user of a Hogwild epoch, by one warp. `ring` is the warp's
// hog_ring_floats(ST, Fs) floats of shared memory: ST staging slots (q row,
// q^f row, four item-side scalars) followed by a window of kRecWindow of the
// user's rating records. Ratings are staged ST - 1 ahead.
//
// The user-side updates use x - lr (g + reg x) = (1 - lr reg) x - lr g, with
// the constant factor hoisted out of the rating loop; the item-side deltas
// likewise. Same arithmetic as the reference up to FP32 rounding.
template <int VPL, int ST = kStages>
__device__ __forceinline__ void hog_user(const DeviceState& s, const EpochParams& p, uint32_t u, float* ring,
                                         int lane) {
    constexpr int AH = ST - 1;
    const uint32_t Fs = s.Fs, T = s.T, NF = s.NF;
    const uint32_t slot_f = 2 * Fs + kSlotScalars;  // q row, q^f row, scalars
    Rec* recw = reinterpret_cast<Rec*>(ring + (size_t)ST * slot_f);
    const uint64_t start = s.user_off[u], end = s.user_off[u + 1];
    if (start == end) return;
    const uint64_t n = end - start;
    const Rec* rr = s.rec + start;
    const uint64_t ps = s.pr_off[u], pe_ = s.pr_off[u + 1];
    const uint64_t total = n + (p.full_su ? (pe_ - ps) : 0);
    const float norm = sqrtf((float)total);

    // ---- su (src/tx.rs:800-822), from the current y
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
    float bb0 = lane < (int)T ? __ldcg(s.but_bin + (size_t)u * T + lane) : 0.0f;
    float bb1 = lane + 32 < (int)T ? __ldcg(s.but_bin + (size_t)u * T + 32 + lane) : 0.0f;
    float sum_err = 0.0f;
    const float gb = s.gbias;
    const float a_u = 1.0f - p.lr_u * p.reg_u, a_u2 = 1.0f - p.lr_u2 * p.reg_u2;
    const float k_i = -(p.lr_i * p.reg_i), k_qf = -(p.lr_iqf * p.reg_iqf);

    // record window: recw[k % kRecWindow] holds record k for k in [wb, wb + kRecWindow)
    __syncwarp();  // the ring is reused from the previous user
    for (uint32_t k = lane; k < kRecWindow && k < n; k += 32) recw[k] = load_rec(rr + k);
    uint64_t wb = 0;
    __syncwarp();
    // ubias_day pipeline (lane 0): values and (user, day) indices of ratings t..t+AH
    float bq[AH + 1];
    uint32_t dq[AH + 1];
#pragma unroll
    for (int a = 0; a <= AH; ++a) {
        bq[a] = 0.0f;
        dq[a] = 0xffffffffu;
    }
    auto shift = [&]() {
#pragma unroll
        for (int a = 0; a < AH; ++a) {
            bq[a] = bq[a + 1];
            dq[a] = dq[a + 1];
        }
    };

    auto issue = [&](uint64_t t) {
        if (t < n) {
            if (t == wb + kRecWindow) {
                // records t .. t+31 replace wb .. wb+31, all consumed by now
                __syncwarp();
                if (t + lane < n) recw[(t + lane) % kRecWindow] = load_rec(rr + t + lane);
                wb += 32;
                __syncwarp();
            }
            const Rec r = recw[t % kRecWindow];
            const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
            const bool hud = r.ud < s.n_ud;
            float* slot = ring + (size_t)(t % ST) * slot_f;
            row_cp_async<VPL>(slot, s.ifeat + (size_t)i * Fs, lane);
            row_cp_async<VPL>(slot + Fs, s.ifeat_freq + (size_t)i * NF * Fs, lane);
            if (lane < 4) {
                const float* src = lane == 0   ? s.ibias + i
                                   : lane == 1 ? s.bit_bin + (size_t)i * T + tb
                                   : lane == 2 ? s.ibias_freq + (size_t)i * NF
                                               : s.cut + (hud ? r.ud : 0u);
                cp_async4(slot + 2 * Fs + lane, src);
            }
            float bnew = 0.0f;
            if (lane == 0 && hud) bnew = s.ubias_day[r.ud];
            bq[AH] = bnew;
            dq[AH] = r.ud;
        }
        cp_async_commit();
    };
    // prologue: ratings 0..AH-1, shifted into the b/d pipeline
#pragma unroll
    for (int a = 0; a < AH; ++a) {
        issue((uint64_t)a);
        shift();
    }
    for (uint64_t t = 0; t < n; ++t) {
        __syncwarp();
        issue(t + AH);
        cp_async_wait<AH>();
        __syncwarp();
        const float* slot = ring + (size_t)(t % ST) * slot_f;
        float q[VPL], qf[VPL];
        row_from_smem<VPL>(slot, lane, q);
        row_from_smem<VPL>(slot + Fs, lane, qf);
        const float4 scv = *reinterpret_cast<const float4*>(slot + 2 * Fs);
        const Rec r = recw[t % kRecWindow];
        const uint32_t i = rec_id(r.key), tb = rec_tbin(r.key);
        const uint32_t ud = r.ud;
        const bool hud = ud < s.n_ud;
        const float dv = r.dev;
        const float ib = scv.x, bit = scv.y, ibf = scv.z, ct = hud ? scv.w : 0.0f;
        const float bud = __shfl_sync(kFull, bq[0], 0);
        const float but = __shfl_sync(kFull, tb < 32 ? bb0 : bb1, tb & 31);
        const float bu_t = ub + but + al * dv + bud + sub;
        const float bi_t = ib + bit + ibf;
        const float cu_t = cuu + ct;
        float part = 0.0f;
#pragma unroll
        for (int v = 0; v < VPL; ++v) part += (q[v] + qf[v]) * ((pu[v] + su[v]) + dv * p2[v]);
        const float dot = warp_sum(part);
        const float score = gb + bu_t + bi_t * cu_t + dot;
        // err = score - r, or the ordinal head's d(-log P)/d(score) (src/tx.rs:963-972)
        float err = score - r.res;
        if (s.raw) {  // thresholds are constant while lr_t = 0
            const float th[4] = {__ldg(s.thresholds), __ldg(s.thresholds + 1), __ldg(s.thresholds + 2),
                                 __ldg(s.thresholds + 3)};
            err = ordinal_grad(th, score, (int)__ldg(s.raw + start + t));
        }
        const float err_b = err * p.w_bias, err_d = err * p.w_factor;
        ub -= p.lr_ub * err_b;
        {
            const float nb = but - p.lr_tu * err_b;
            if (lane == (int)(tb & 31)) {
                if (tb < 32) bb0 = nb;
                else bb1 = nb;
            }
        }
        al -= p.lr_ta * err_b * dv;
        if (lane == 0 && hud) {
            const float nv = bud - p.lr_ubd * err_b;
            s.ubias_day[ud] = nv;
#pragma unroll
            for (int a = 1; a <= AH; ++a)
                if (dq[a] == ud) bq[a] = nv;
        }
        if (lane == 0) {
            // item-side updates are applied as atomic deltas: users that
            // run concurrently never overwrite each other's update
            const float ge = err_b * cu_t;
            atomicAdd(s.ibias + i, -(p.lr_ib * ge));
            atomicAdd(s.bit_bin + (size_t)i * T + tb, -(p.lr_ti * ge));
            atomicAdd(s.ibias_freq + (size_t)i * NF, -(p.lr_ibf * ge));
        }
        cuu -= p.lr_cu * (err_b * bi_t + p.reg_cu * (cuu - 1.0f));
        if (!p.sum_err_bug) sum_err += err_b;
        else
            for (uint32_t kk = 0; kk < s.F; ++kk) sum_err += err_b;
        const float nlu = -(p.lr_u * err_d), nlu2 = -(p.lr_u2 * err_d) * dv;
        const float nli = -(p.lr_i * err_d), nlf = -(p.lr_iqf * err_d);
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
            const float qe = q[v] + qf[v];
            const float pk = pu[v], p2k = p2[v];
            seq[v] += err_d * qe;
            pu[v] = fmaf(nlu, qe, a_u * pk);
            p2[v] = fmaf(nlu2, qe, a_u2 * p2k);
            const float pe = fmaf(dv, p2k, pk) + su[v];
            q[v] = fmaf(nli, pe, k_i * q[v]);     // delta of q_i
            qf[v] = fmaf(nlf, pe, k_qf * qf[v]);  // delta of q^f_i
        }
        Row<VPL>::red_add(s.ifeat + (size_t)i * Fs, lane, q);
        Row<VPL>::red_add(s.ifeat_freq + (size_t)i * NF * Fs, lane, qf);
        shift();
    }
    cp_async_wait<0>();

    Row<VPL>::store(s.ufeat + (size_t)u * Fs, lane, pu);
    Row<VPL>::store(s.ufeat2 + (size_t)u * Fs, lane, p2);
    if (lane == 0) {
        s.ubias[u] = ub;
        s.alpha_u[u] = al;
        s.cu[u] = cuu;
    }
    if (lane < (int)T) s.but_bin[(size_t)u * T + lane] = bb0;
    if (lane + 32 < (int)T) s.but_bin[(size_t)u * T + 32 + lane] = bb1;

    // ---- NSVD1 factor & bias updates at the end of the user (src/tx.rs:1099-1106)
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
}

template <int VPL>
__global__ void __launch_bounds__(kThreads, 2) k_hog_pass(DeviceState s, EpochParams p,
                                                          const uint32_t* __restrict__ order, uint32_t n_work) {
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* ring = smem + (size_t)warp * hog_ring_floats(kStages, s.Fs);
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&s.counters[0], 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= n_work) break;
        hog_user<VPL>(s, p, order[k], ring, lane);
    }
}

// Out-of-line entry for the batched kernel: each (VPL, ring depth) instance
// keeps its own register allocation (the call costs once per user, not per
// rating).
template <int VPL, int ST>
__device__ __noinline__ void hog_user_st(const DeviceState* s, const EpochParams* p, uint32_t u, float* ring,
                                         int lane) {
    hog_user<VPL, ST>(*s, *p, u, ring, lane);
}

template <int VPL>
__device__ __forceinline__ void hog_user_call(const DeviceState* s, const EpochParams* p, uint32_t u, float* ring,
                                              int lane) {
    const int st = p->stages;
    if (st == 2) hog_user_st<VPL, 2>(s, p, u, ring, lane);
    else if (st == 3) hog_user_st<VPL, 3>(s, p, u, ring, lane);
    else hog_user_st<VPL, 4>(s, p, u, ring, lane);
}

// ---------------------------------------------------------------------------
// Batched Hogwild epoch: several model variants over one dataset in a single
// persistent launch. A work unit is (variant, user), packed as
// variant << 24 | user; units of the same user for every variant are adjacent,
// so a user's rating records are read while still in L2. Each unit runs the
// variant's VPL instance of hog_user; the shared-memory ring is sized for the
// widest variant.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2) k_hog_batched(const DeviceState* __restrict__ states,
                                                             const EpochParams* __restrict__ params,
                                                             const uint32_t* __restrict__ units, uint32_t n_units,
                                                             uint32_t ring_floats, uint32_t* __restrict__ counter) {
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* ring = smem + (size_t)warp * ring_floats;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(counter, 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= n_units) break;
        const uint32_t unit = units[k];
        const uint32_t mk = unit >> 24, u = unit & 0xffffffu;
        const DeviceState* s = states + mk;
        const EpochParams* p = params + mk;
        switch (s->Fs >> 5) {
            case 1: hog_user_call<1>(s, p, u, ring, lane); break;
            case 2: hog_user_call<2>(s, p, u, ring, lane); break;
            case 3: hog_user_call<3>(s, p, u, ring, lane); break;
            case 4: hog_user_call<4>(s, p, u, ring, lane); break;
            case 5: hog_user_call<5>(s, p, u, ring, lane); break;
            case 6: hog_user_call<6>(s, p, u, ring, lane); break;
            case 7: hog_user_call<7>(s, p, u, ring, lane); break;
            default: hog_user_call<8>(s, p, u, ring, lane); break;
        }
    }
}


// ---------------------------------------------------------------------------
// ycache[u] = |N(u)|^-1/2 sum over train and pr items (rebuild_ycache,
// src/tx.rs:391-418): train items in rating order, then pr items in pr order.
// ---------------------------------------------------------------------------
template <int VPL>
__global__ void __launch_bounds__(kThreads) k_rebuild_ycache(DeviceState s, const __nv_bfloat16* __restrict__ ybf,
                                                              float* __restrict__ pyc);

template <int VPL>
__device__ __forceinline__ void rebuild_user(const DeviceState& s, const __nv_bfloat16* __restrict__ ybf, uint32_t u,
                                             int lane, float* __restrict__ pyc) {
    constexpr int B = 8;  // rows in flight
    const uint64_t a = s.user_off[u], b = s.user_off[u + 1];
    const uint64_t pa = s.pr_off[u], pb = s.pr_off[u + 1];
    const uint64_t ntr = b - a, n = ntr + (pb - pa);
    const int32_t cnt_all = s.user_cnt_tr[u] + s.user_cnt_pr[u];
    // rows wider than 32 * VPL columns (n_feat > 256) in slices of 32 * VPL
    for (uint32_t c0 = 0; c0 < s.Fs; c0 += 32 * VPL) {
        float su[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) su[v] = 0.0f;
        float sub = 0.0f;
        // the item of entry q of N(u): training ratings first, then pr items
        auto item_at = [&](uint64_t q) -> uint32_t {
            return q < ntr ? rec_id(__ldg(&s.rec[a + q].key)) : __ldg(s.pr_item + pa + (q - ntr));
        };
        // each chunk's 32 items are loaded one chunk ahead (one per lane)
        uint32_t nxt = (uint64_t)lane < n ? item_at(lane) : 0u;
        for (uint64_t base = 0; base < n; base += 32) {
            const uint32_t cnt = (uint32_t)(n - base < 32 ? n - base : 32);
            const uint32_t mine = nxt;
            if (base + 32 + lane < n) nxt = item_at(base + 32 + lane);
            for (uint32_t j = 0; j < cnt; j += B) {
                float y[B][VPL], yb[B];
#pragma unroll
                for (int t = 0; t < B; ++t) {
                    const uint32_t it = __shfl_sync(kFull, mine, j + t < cnt ? j + t : cnt - 1);
                    if (ybf) row_load_bf16<VPL>(ybf + (size_t)it * s.Fs + c0, lane, y[t]);
                    else Row<VPL>::load_nc(s.yfeat + (size_t)it * s.Fs + c0, lane, y[t]);
                    yb[t] = c0 == 0 ? __ldg(s.ybias + it) : 0.0f;
                }
#pragma unroll
                for (int t = 0; t < B; ++t) {
                    if (j + t < cnt) {
#pragma unroll
                        for (int v = 0; v < VPL; ++v) su[v] += y[t][v];
                        sub += yb[t];
                    }
                }
            }
        }
        if (cnt_all > 0) {
            const float nrm = sqrtf((float)cnt_all);
#pragma unroll
            for (int v = 0; v < VPL; ++v) su[v] = su[v] / nrm;
            sub = sub / nrm;
        }
        Row<VPL>::store(s.ycache + (size_t)u * s.Fs + c0, lane, su);
        if (lane == 0 && c0 == 0) s.ycache_bias[u] = sub;
        if (pyc) {
            // p_u + ycache_u, the user-side sum every item-stratum rating of u reads
            float pu[VPL];
            Row<VPL>::load_cg(s.ufeat + (size_t)u * s.Fs + c0, lane, pu);
#pragma unroll
            for (int v = 0; v < VPL; ++v) pu[v] = pu[v] + su[v];
            Row<VPL>::store(pyc + (size_t)u * s.Fs + c0, lane, pu);
        }
    }
}

// Batched ycache rebuild over (variant, user) pairs, variant-major.
__global__ void __launch_bounds__(kThreads) k_rebuild_batched(const DeviceState* __restrict__ states,
                                                              uint32_t n_models, uint32_t n_users) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * kWarps;
    const uint64_t total = (uint64_t)n_models * n_users;
    for (uint64_t w = blockIdx.x * (uint64_t)kWarps + (threadIdx.x >> 5); w < total; w += warps) {
        const uint32_t mk = (uint32_t)(w / n_users), u = (uint32_t)(w - (uint64_t)mk * n_users);
        const DeviceState& s = states[mk];
        switch (s.Fs >> 5) {
            case 1: rebuild_user<1>(s, nullptr, u, lane, nullptr); break;
            case 2: rebuild_user<2>(s, nullptr, u, lane, nullptr); break;
            case 3: rebuild_user<3>(s, nullptr, u, lane, nullptr); break;
            case 4: rebuild_user<4>(s, nullptr, u, lane, nullptr); break;
            case 5: rebuild_user<5>(s, nullptr, u, lane, nullptr); break;
            case 6: rebuild_user<6>(s, nullptr, u, lane, nullptr); break;
            case 7: rebuild_user<7>(s, nullptr, u, lane, nullptr); break;
            default: rebuild_user<8>(s, nullptr, u, lane, nullptr); break;
        }
    }
}

template <int VPL>
__global__ void __launch_bounds__(kThreads) k_rebuild_ycache(DeviceState s, const __nv_bfloat16* __restrict__ ybf,
                                                              float* __restrict__ pyc) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * kWarps;
    for (uint32_t u = blockIdx.x * kWarps + (threadIdx.x >> 5); u < s.n_users; u += warps)
        rebuild_user<VPL>(s, ybf, u, lane, pyc);
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <int VPL>
void launch_hog_pass(tsvd_model* m, const EpochParams& p, const uint32_t* order) {
    const size_t smem = (size_t)kWarps * hog_ring_floats(kStages, m->d.Fs) * sizeof(float);
    TSVD_CUDA(cudaFuncSetAttribute(k_hog_pass<VPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    unsigned g = persistent_grid(k_hog_pass<VPL>, smem);
    k_hog_pass<VPL><<<g, kThreads, smem, m->stream>>>(m->d, p, order, m->d.n_users);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

template <int VPL>
void launch_rebuild(tsvd_model* m, const __nv_bfloat16* ybf, float* pyc) {
    unsigned g = persistent_grid(k_rebuild_ycache<VPL>, 0);
    k_rebuild_ycache<VPL><<<g, kThreads, 0, m->stream>>>(m->d, ybf, pyc);
    TSVD_CUDA(cudaGetLastError());
    m->launches++;
}

}  // namespace

void launch_hog_batched(cudaStream_t st, const DeviceState* d_states, const EpochParams* d_params,
                        const uint32_t* d_units, uint32_t n_units, uint32_t ring_floats, uint32_t* d_counter) {
    const size_t smem = (size_t)kWarps * ring_floats * sizeof(float);
    TSVD_CUDA(cudaFuncSetAttribute(k_hog_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    unsigned g = persistent_grid(k_hog_batched, smem);
    k_hog_batched<<<g, kThreads, smem, st>>>(d_states, d_params, d_units, n_units, ring_floats, d_counter);
    TSVD_CUDA(cudaGetLastError());
}

void launch_rebuild_batched(cudaStream_t st, const DeviceState* d_states, uint32_t n_models, uint32_t n_users) {
    unsigned g = persistent_grid(k_rebuild_batched, 0);
    k_rebuild_batched<<<g, kThreads, 0, st>>>(d_states, n_models, n_users);
    TSVD_CUDA(cudaGetLastError());
}

namespace {

void reset_counters(tsvd_model* m) {
    TSVD_CUDA(cudaMemsetAsync(m->d.counters, 0, 64, m->stream));
}

}  // namespace

// Rebuild from the FP32 masters (explicit calls, Hogwild epochs).
void rebuild_ycache(tsvd_model* m) {
    ProfScope ps(m, "rebuild_ycache");
    const int vpl = (int)std::min<uint32_t>(m->d.Fs / 32, 8);
    TSVD_DISPATCH(vpl, launch_rebuild<V>(m, nullptr, nullptr));
    m->ycache_valid = true;
}

// Rebuild inside a stratified epoch: from the BF16 read copy of y in the
// precision form, else from the FP32 master.
void launch_rebuild_ycache(tsvd_model* m, float* pyc) {
    ProfScope ps(m, "rebuild_ycache");
    const __nv_bfloat16* ybf =
        m->opts.precision >= TSVD_PREC_BF16_READ ? m->m_bf_yfeat.as<__nv_bfloat16>() : nullptr;
    const int vpl = (int)std::min<uint32_t>(m->d.Fs / 32, 8);
    TSVD_DISPATCH(vpl, launch_rebuild<V>(m, ybf, pyc));
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
    // Tsvdx4pModel::fit_epoch runs TxModel::fit_epoch on its seq_epochs
    // (src/tsvdx4p.rs:815-822)
    bool seq_now = m->opts.schedule == TSVD_SCHED_SEQUENTIAL;
    if (m->opts.schedule == TSVD_SCHED_STRATIFIED)
        for (int k = 0; k < 5; ++k)
            if (m->opts.seq_epochs[k] > 0 && (uint64_t)m->opts.seq_epochs[k] == epoch) seq_now = true;
    if (m->opts.schedule == TSVD_SCHED_HOGWILD || seq_now) {
        // per-epoch user order: injected, or get_users (src/lib.rs:486-494)
        std::vector<uint32_t> order;
        auto it = m->injected_order.find(epoch);
        if (it != m->injected_order.end()) order = it->second;
        else order = user_order(m->d.n_users, c.shuffle_users != 0, c.seed, epoch);
        TSVD_CUDA(cudaMemcpyAsync(m->m_perm.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));  // `order` leaves scope
        if (seq_now || !c.low_memory) {
            day_epoch_pass(m, m->m_perm.as<uint32_t>(), seq_now);
        } else {
            ProfScope ps(m, "user_pass_hogwild");
            TSVD_DISPATCH(vpl, launch_hog_pass<V>(m, p, m->m_perm.as<uint32_t>()));
        }
        rebuild_ycache(m);
        rebuild_ycache_day(m);
        if (c.has_ordinal_head && c.ordinal_head.lr_t != 0.0f) {
            // thresholds moved on the device during the pass
            TSVD_CUDA(cudaMemcpyAsync(m->h_thresholds, m->d.thresholds, 16, cudaMemcpyDeviceToHost, m->stream));
            TSVD_CUDA(cudaStreamSynchronize(m->stream));
        }
    } else {
        p.use_ycache = (c.full_su && m->ycache_valid) ? 1 : 0;
        stratified_epoch(m, p);
    }
    finish_epoch(m);
}

void finish_epoch(tsvd_model* m) {
    const tsvd_config& c = m->cfg;
    if (c.has_ordinal_head) {
        // OrdinalHead::enforce_sorted_with_gap at the end of the epoch
        // (src/tx.rs:1112-1114, src/lib.rs:518-525)
        float* th = m->h_thresholds;
        std::sort(th, th + 4);
        for (int k = 1; k < 4; ++k) {
            const float min_ok = th[k - 1] + c.ordinal_head.th_gap;
            if (th[k] < min_ok) th[k] = min_ok;
        }
        TSVD_CUDA(cudaMemcpyAsync(m->d.thresholds, th, 16, cudaMemcpyHostToDevice, m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    }
}

}  // namespace tsvd
