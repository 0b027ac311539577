// Model construction: the device-side counterpart of TxModel::new
// (src/tx.rs:460-649) plus the one-time per-rating precompute that the
// reference repeats inside every epoch (time_bin, dev and the SparseUD
// binary search at src/tx.rs:841-842,878; freq_bin at :851).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "rand_stream.hpp"
#include "tsvd_device.cuh"

namespace tsvd {
namespace {

__global__ void k_ud_keys(const int32_t* __restrict__ u, const int16_t* __restrict__ d, uint64_t n,
                          uint64_t* __restrict__ keys) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x)
        keys[t] = ((uint64_t)(uint32_t)u[t] << 16) | (uint64_t)(uint16_t)((int32_t)d[t] + 32768);
}

__global__ void k_ud_split(const uint64_t* __restrict__ ukeys, const uint32_t* __restrict__ cnts, uint64_t n_ud,
                           int16_t* __restrict__ date, uint32_t* __restrict__ cnt_out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_ud; k += (uint64_t)gridDim.x * blockDim.x) {
        date[k] = (int16_t)((int32_t)(ukeys[k] & 0xffff) - 32768);
        cnt_out[k] = cnts[k];
    }
}

// start[u] = first k with user(key[k]) >= u, for u in [0, U].
__global__ void k_lower_bound_users(const uint64_t* __restrict__ ukeys, uint64_t n, uint32_t U,
                                    uint64_t* __restrict__ start) {
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u <= U; u += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = n, target = u << 16;
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (ukeys[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        start[u] = lo;
    }
}

__global__ void k_records(DeviceState s, const int32_t* __restrict__ u, const int32_t* __restrict__ it,
                          const int16_t* __restrict__ d, const float* __restrict__ res, float beta,
                          Rec* __restrict__ out) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < s.n_train;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t uu = (uint32_t)u[t];
        int16_t day = d[t];
        uint32_t tb = time_bin(day, s.day_range, s.T);
        uint32_t ud = ud_index(s, uu, day);
        uint32_t fb = ud == 0xffffffffu ? 0u : freq_bin(s.ud_cnt[ud], s.NF);
        Rec r;
        r.key = ((uint32_t)it[t] & kIdMask) | (tb << 20) | (fb << 26);
        r.res = res[t];
        r.dev = dev_of(day, s.tu_mean[uu], beta);
        r.ud = ud;
        out[t] = r;
    }
}

__global__ void k_item_records(const Rec* __restrict__ rec, const int32_t* __restrict__ u,
                               const uint32_t* __restrict__ order, uint64_t n, Rec* __restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t t = order[k];
        Rec r = rec[t];
        r.key = ((uint32_t)u[t] & kIdMask) | (r.key & ~kIdMask);
        out[k] = r;
    }
}

__global__ void k_gather_u32(const int32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint64_t n,
                             uint32_t* __restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = (uint32_t)src[idx[k]];
}

__global__ void k_iota(uint32_t* __restrict__ v, uint64_t n) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        v[k] = (uint32_t)k;
}

// off[j] = the first position t of the sorted keys with key >= j (j = 0..I),
// so item j's entries are off[j] .. off[j+1]-1; each j is written once.
__global__ void k_item_offsets(const uint32_t* __restrict__ sorted, uint64_t R, uint32_t I, uint64_t* __restrict__ off) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t <= R; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = t == 0 ? 0u : sorted[t - 1] + 1u;
        const uint32_t b = t == R ? I : sorted[t];
        for (uint32_t j = a; j <= b; ++j) off[j] = t;
    }
}

__global__ void k_fill(float* __restrict__ v, uint64_t n, float x) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        v[k] = x;
}

// (user, day) keys of the per-ud item lists: pr rows first (pr order), then
// training rows (training order); values are the items. Counts pr rows per ud.
__global__ void k_ud_list_keys(DeviceState s, const int32_t* __restrict__ pu, const int32_t* __restrict__ pi,
                               const int16_t* __restrict__ pd, uint64_t P, uint32_t* __restrict__ key,
                               uint32_t* __restrict__ val, uint32_t* __restrict__ pr_cnt) {
    const uint64_t n = P + s.n_train;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        if (k < P) {
            const uint32_t ud = ud_index(s, (uint32_t)pu[k], pd[k]);  // present: SparseUD covers pr
            key[k] = ud;
            val[k] = (uint32_t)pi[k];
            atomicAdd(pr_cnt + ud, 1u);
        } else {
            const Rec r = s.rec[k - P];
            key[k] = r.ud;
            val[k] = rec_id(r.key);
        }
    }
}

// off[d] = first k with keys[k] >= d, for d in [0, n_ud].
__global__ void k_lower_bound_u32(const uint32_t* __restrict__ keys, uint64_t n, uint64_t n_ud,
                                  uint64_t* __restrict__ off) {
    for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d <= n_ud; d += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < d) lo = mid + 1;
            else hi = mid;
        }
        off[d] = lo;
    }
}

constexpr unsigned kGrid = 148 * 8, kBlock = 256;

template <class T>
void upload(DevMem& m, const T* src, size_t n, cudaStream_t st) {
    m.alloc(n * sizeof(T));
    if (n) TSVD_CUDA(cudaMemcpyAsync(m.p, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

void zeros(DevMem& m, size_t bytes, cudaStream_t st) {
    m.alloc(bytes);
    TSVD_CUDA(cudaMemsetAsync(m.p, 0, m.bytes, st));
}

// Stable radix sort of (key, value) pairs over the low `bits` key bits.
template <class K>
void sort_pairs(DevMem& tmp, const K* kin, K* kout, const uint32_t* vin, uint32_t* vout, uint64_t n, int bits,
                cudaStream_t st) {
    size_t need = 0;
    TSVD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, kin, kout, vin, vout, (int64_t)n, 0, bits, st));
    if (tmp.bytes < need) tmp.alloc(need);
    size_t have = tmp.bytes;
    TSVD_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, have, kin, kout, vin, vout, (int64_t)n, 0, bits, st));
}

int bits_for(uint64_t maxv) {
    int b = 1;
    while (b < 64 && (maxv >> b) != 0) ++b;
    return b;
}

}  // namespace

// 0 .. n-1 ordered by count, largest first, ties in index order: a stable
// counting sort, the same order as a stable sort by descending count.
template <class C>
std::vector<uint32_t> heaviest_first(const C* cnt, uint32_t n) {
    uint64_t mx = 0;
    for (uint32_t i = 0; i < n; ++i) mx = std::max<uint64_t>(mx, (uint64_t)cnt[i]);
    std::vector<uint32_t> start(mx + 2, 0u);
    for (uint32_t i = 0; i < n; ++i) start[mx - (uint64_t)cnt[i] + 1]++;
    for (uint64_t b = 1; b < start.size(); ++b) start[b] += start[b - 1];
    std::vector<uint32_t> out(n);
    for (uint32_t i = 0; i < n; ++i) out[start[mx - (uint64_t)cnt[i]]++] = i;
    return out;
}

void setup_model(tsvd_model* m, const tsvd_dataset_view& tr, const tsvd_dataset_view& pr) {
    const tsvd_config& c = m->cfg;
    cudaStream_t st = m->stream;
    DeviceState& s = m->d;
    // ---- validation (the reference panics on the same conditions) ----------
    if (!tr.user_idxs || !tr.item_idxs || !tr.residuals || !tr.dates || !tr.user_cnts)
        throw Error(TSVD_ERR_INVALID, "training view lacks user_idxs/item_idxs/residuals/dates/user_cnts");
    if (!pr.user_idxs || !pr.item_idxs || !pr.dates || !pr.user_cnts)
        throw Error(TSVD_ERR_INVALID, "pr view lacks user_idxs/item_idxs/dates/user_cnts");
    if (pr.n_users != tr.n_users) throw Error(TSVD_ERR_INVALID, "train and pr disagree on n_users");
    if (c.lr_w != 0 || c.lr_c != 0 || c.lr_w_day != 0 || c.lr_c_day != 0)
        throw Error(TSVD_ERR_UNSUPPORTED, "neighbourhood terms (tx5/tx6) are outside the tsvdx4 path");
    if (c.n_feat > (1u << 16)) throw Error(TSVD_ERR_UNSUPPORTED, "n_feat must be at most 65536");
    if (c.n_feat > 256) {
        // wide rows: the stratified and sequential schedules, low_memory, FP32
        // (every tsvdx4 / tsvdx4p job above 256 factors, src/bin/tsvdx4-new.rs:19-22,
        // src/bin/tsvdx4p-new.rs:14-19)
        if (m->opts.schedule == TSVD_SCHED_HOGWILD)
            throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256 runs with the stratified or sequential schedule");
        if (!c.low_memory) throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256 is built for low_memory = true");
        if (c.has_ordinal_head) throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256 is built without the ordinal head");
        if (m->opts.precision != TSVD_PREC_FP32)
            throw Error(TSVD_ERR_UNSUPPORTED, "n_feat above 256 is built for FP32 reads");
    }
    if (c.n_time_bins < 1 || c.n_time_bins > kMaxBins) throw Error(TSVD_ERR_UNSUPPORTED, "n_time_bins must be in 1..64");
    if (c.n_freq_bins < 1 || c.n_freq_bins > kMaxBins) throw Error(TSVD_ERR_UNSUPPORTED, "n_freq_bins must be in 1..64");
    if (tr.n_users == 0 || tr.n_users > (1u << kIdBits) || tr.n_items == 0 || tr.n_items > (1u << kIdBits))
        throw Error(TSVD_ERR_UNSUPPORTED, "n_users and n_items must be in 1..2^20");
    if (tr.n_ratings == 0) throw Error(TSVD_ERR_INVALID, "empty training set");
    if (tr.n_ratings >= (1ull << 32) || pr.n_ratings >= (1ull << 32))
        throw Error(TSVD_ERR_UNSUPPORTED, "at most 2^32-1 ratings per set");
    if (!c.low_memory && m->opts.precision != TSVD_PREC_FP32)
        throw Error(TSVD_ERR_UNSUPPORTED, "BF16 read copies are built for low_memory = true");
    for (int k = 0; k < 5; ++k) {
        if (m->opts.seq_epochs[k] < 0) throw Error(TSVD_ERR_INVALID, "seq_epochs entries must be >= 0");
        if (m->opts.seq_epochs[k] > 0 && m->opts.schedule != TSVD_SCHED_STRATIFIED)
            throw Error(TSVD_ERR_INVALID, "seq_epochs belong to the stratified schedule");
    }
    if (c.has_ordinal_head) {
        // The reference moves the 4 shared thresholds after every rating
        // (src/tx.rs:965-969), a serial chain over the whole epoch; every
        // tsvdx4 job sets lr_t = 0, which every schedule runs (the thresholds
        // then only shape the error and the prediction).
        if (c.ordinal_head.lr_t != 0.0f && m->opts.schedule != TSVD_SCHED_SEQUENTIAL)
            throw Error(TSVD_ERR_UNSUPPORTED,
                        "ordinal head with lr_t != 0 (thresholds trained per rating) needs the sequential schedule");
        if (!tr.raw_ratings) throw Error(TSVD_ERR_INVALID, "the ordinal head needs the training raw_ratings");
        for (uint64_t t = 0; t < tr.n_ratings; ++t)
            if (tr.raw_ratings[t] < 1 || tr.raw_ratings[t] > 5)
                throw Error(TSVD_ERR_INVALID, "ordinal head: training rating outside 1..5");
    }

    const uint32_t U = (uint32_t)tr.n_users, I = (uint32_t)tr.n_items;
    const uint64_t R = tr.n_ratings, P = pr.n_ratings;
    // The raw columns go up first, so that the copies (asynchronous from pinned
    // buffers) overlap the host-side checks and sums below; nothing on the
    // device reads them before those checks have passed.
    DevMem d_tu, d_ti, d_td, d_tres, d_pu, d_pi, d_pd, tmp;
    upload(d_tu, tr.user_idxs, R, st);
    upload(d_ti, tr.item_idxs, R, st);
    upload(d_td, tr.dates, R, st);
    if (!c.has_ordinal_head) upload(d_tres, tr.residuals, R, st);
    upload(d_pu, pr.user_idxs, P, st);
    upload(d_pi, pr.item_idxs, P, st);
    upload(d_pd, pr.dates, P, st);
    // calc_user_offsets (src/lib.rs:470-483): user-sorted, offsets from user_cnts.
    std::vector<uint64_t> uoff(U + 1, 0);
    for (uint32_t u = 0; u < U; ++u) {
        if (tr.user_cnts[u] < 0) throw Error(TSVD_ERR_INVALID, "negative user count");
        uoff[u + 1] = uoff[u] + (uint64_t)tr.user_cnts[u];
    }
    if (uoff[U] != R) throw Error(TSVD_ERR_INVALID, "training user_cnts do not sum to n_ratings");
    // Every rating of user u lies in uoff[u] .. uoff[u+1] and its item is in
    // range: checked over users in parallel; a failure reruns the checks in
    // rating order for the reference's message.
    bool rows_ok = true;
#pragma omp parallel for schedule(dynamic, 4096) reduction(&& : rows_ok)
    for (int64_t uu = 0; uu < (int64_t)U; ++uu) {
        for (uint64_t t = uoff[uu]; t < uoff[uu + 1]; ++t) {
            const int32_t i = tr.item_idxs[t];
            rows_ok = rows_ok && tr.user_idxs[t] == (int32_t)uu && i >= 0 && (uint32_t)i < I;
        }
    }
    if (!rows_ok) {
        uint32_t prev = 0;
        for (uint64_t t = 0; t < R; ++t) {
            int32_t u = tr.user_idxs[t];
            if (u < 0 || (uint32_t)u >= U) throw Error(TSVD_ERR_INVALID, "training user index out of range");
            if ((uint32_t)u < prev)
                throw Error(TSVD_ERR_INVALID, "training set is not user-sorted at index " + std::to_string(t));
            prev = (uint32_t)u;
            int32_t i = tr.item_idxs[t];
            if (i < 0 || (uint32_t)i >= I) throw Error(TSVD_ERR_INVALID, "training item index out of range");
        }
        throw Error(TSVD_ERR_INVALID, "training user_cnts disagree with user_idxs");
    }
    {
        std::vector<int64_t> pcnt(U, 0);
        for (uint64_t t = 0; t < P; ++t) {
            int32_t u = pr.user_idxs[t], i = pr.item_idxs[t];
            if (u < 0 || (uint32_t)u >= U || i < 0 || (uint32_t)i >= I)
                throw Error(TSVD_ERR_INVALID, "pr index out of range");
            pcnt[u]++;
        }
        for (uint32_t u = 0; u < U; ++u)
            if (pcnt[u] != pr.user_cnts[u]) throw Error(TSVD_ERR_INVALID, "pr user_cnts disagree with user_idxs");
    }
    // tu_mean in f32, summed in rating order; day_range; gbias (src/tx.rs:465-475,
    // src/lib.rs:463-467). Users in parallel: a user's dates add in rating
    // order, so tu_mean is the reference's; the FP64 residual sum adds the
    // users' sums in user order (exact for integer residuals).
    std::vector<float> tum(U, 0.0f);
    std::vector<double> usum(U, 0.0);
    int32_t dr = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(max : dr)
    for (int64_t uu = 0; uu < (int64_t)U; ++uu) {
        float a = 0.0f;
        double b = 0.0;
        for (uint64_t t = uoff[uu]; t < uoff[uu + 1]; ++t) {
            a += (float)tr.dates[t];
            dr = std::max(dr, (int32_t)tr.dates[t] + 1);
            b += (double)tr.residuals[t];
        }
        tum[uu] = tr.user_cnts[uu] > 0 ? a / (float)tr.user_cnts[uu] : a;
        usum[uu] = b;
    }
    double rsum = 0.0;
    for (uint32_t u = 0; u < U; ++u) rsum += usum[u];
    if (dr <= 0) throw Error(TSVD_ERR_INVALID, "training dates must include a non-negative day");

    // Rows padded with zeros (which every update keeps at zero): to a multiple
    // of 32 floats up to 256 (a warp's row), of 256 above (slices of a warp's
    // row); n_feat = 0 (bias-only jobs) keeps one all-zero 32-float row.
    const uint32_t F = (uint32_t)c.n_feat;
    const uint32_t Fs = F == 0 ? 32u : F <= 256 ? (F + 31) / 32 * 32 : (F + 255) / 256 * 256;
    s.n_users = U; s.n_items = I; s.F = F; s.Fs = Fs;
    s.T = (uint32_t)c.n_time_bins; s.NF = (uint32_t)c.n_freq_bins;
    // Heavy items run as rounds on a whole block; below the threshold a warp
    // per item is cheaper per rating, as long as its chain stays shorter than
    // the hottest item's (32768 measured best at the full Netflix shape).
    s.heavy_min = m->opts.heavy_item_ratings > 0 ? (uint32_t)m->opts.heavy_item_ratings : 32768u;
    s.n_train = R; s.n_pr = P;
    s.day_range = dr;
    s.gbias = (float)(rsum / (double)R);
    m->h_user_cnt.assign(tr.user_cnts, tr.user_cnts + U);

    // ---- upload raw columns (the rest; see above) ------------------------------
    if (c.has_ordinal_head) {
        // with the head the error comes from the raw rating, not the residual
        // (src/tx.rs:965-969): the records carry the raw rating instead
        std::vector<float> rawf(R);
        for (uint64_t t = 0; t < R; ++t) rawf[t] = (float)tr.raw_ratings[t];
        upload(d_tres, rawf.data(), R, st);
        TSVD_CUDA(cudaStreamSynchronize(st));
    }
    upload(m->m_user_off, uoff.data(), U + 1, st);
    upload(m->m_tu_mean, tum.data(), U, st);
    s.raw = nullptr;
    if (c.has_ordinal_head) {
        upload(m->m_raw, tr.raw_ratings, R, st);
        s.raw = m->m_raw.as<int8_t>();
    }
    upload(m->m_ucnt_tr, tr.user_cnts, U, st);
    upload(m->m_ucnt_pr, pr.user_cnts, U, st);
    s.user_off = m->m_user_off.as<uint64_t>();
    s.tu_mean = m->m_tu_mean.as<float>();
    s.user_cnt_tr = m->m_ucnt_tr.as<int32_t>();
    s.user_cnt_pr = m->m_ucnt_pr.as<int32_t>();

    // ---- SparseUD over train + pr (src/tx.rs:21-84) -------------------------
    {
        DevMem keys, keys_sorted, ukeys, ucnt, nrun;
        keys.alloc((R + P) * 8);
        keys_sorted.alloc((R + P) * 8);
        k_ud_keys<<<kGrid, kBlock, 0, st>>>(d_tu.as<int32_t>(), d_td.as<int16_t>(), R, keys.as<uint64_t>());
        if (P) k_ud_keys<<<kGrid, kBlock, 0, st>>>(d_pu.as<int32_t>(), d_pd.as<int16_t>(), P, keys.as<uint64_t>() + R);
        TSVD_CUDA(cudaGetLastError());
        int kb = 16 + bits_for(U);
        size_t need = 0;
        TSVD_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, need, keys.as<uint64_t>(), keys_sorted.as<uint64_t>(),
                                                 (int64_t)(R + P), 0, kb, st));
        tmp.alloc(need);
        size_t have = tmp.bytes;
        TSVD_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, have, keys.as<uint64_t>(), keys_sorted.as<uint64_t>(),
                                                 (int64_t)(R + P), 0, kb, st));
        ukeys.alloc((R + P) * 8);
        ucnt.alloc((R + P) * 4);
        nrun.alloc(8);
        need = 0;
        TSVD_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, need, keys_sorted.as<uint64_t>(), ukeys.as<uint64_t>(),
                                                     ucnt.as<uint32_t>(), nrun.as<int64_t>(), (int64_t)(R + P), st));
        if (tmp.bytes < need) tmp.alloc(need);
        have = tmp.bytes;
        TSVD_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.p, have, keys_sorted.as<uint64_t>(), ukeys.as<uint64_t>(),
                                                     ucnt.as<uint32_t>(), nrun.as<int64_t>(), (int64_t)(R + P), st));
        int64_t n_ud = 0;
        TSVD_CUDA(cudaMemcpyAsync(&n_ud, nrun.p, 8, cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaStreamSynchronize(st));
        s.n_ud = (uint64_t)n_ud;
        m->m_ud_date.alloc(n_ud * 2);
        m->m_ud_cnt.alloc(n_ud * 4);
        m->m_ud_start.alloc((U + 1) * 8);
        k_ud_split<<<kGrid, kBlock, 0, st>>>(ukeys.as<uint64_t>(), ucnt.as<uint32_t>(), n_ud, m->m_ud_date.as<int16_t>(),
                                             m->m_ud_cnt.as<uint32_t>());
        k_lower_bound_users<<<ceil_div(U + 1, kBlock), kBlock, 0, st>>>(ukeys.as<uint64_t>(), n_ud, U,
                                                                       m->m_ud_start.as<uint64_t>());
        TSVD_CUDA(cudaGetLastError());
        s.ud_start = m->m_ud_start.as<uint64_t>();
        s.ud_date = m->m_ud_date.as<int16_t>();
        s.ud_cnt = m->m_ud_cnt.as<uint32_t>();
        TSVD_CUDA(cudaStreamSynchronize(st));
    }

    // ---- per-rating records (user-major) -------------------------------------
    m->m_rec.alloc(R * sizeof(Rec));
    k_records<<<kGrid, kBlock, 0, st>>>(s, d_tu.as<int32_t>(), d_ti.as<int32_t>(), d_td.as<int16_t>(),
                                        d_tres.as<float>(), c.beta, m->m_rec.as<Rec>());
    TSVD_CUDA(cudaGetLastError());
    s.rec = m->m_rec.as<Rec>();

    // ---- per-(user, day) item lists for the per-day terms (low_memory = false):
    // probe_items_by_ud (src/tx.rs:587-598) and the rebuild_ycache_day order
    // (src/tx.rs:420-454) in one sorted list per ud
    s.ud_list_off = nullptr;
    s.ud_list_item = nullptr;
    s.ud_pr_cnt = nullptr;
    if (!c.low_memory) {
        const uint64_t N = R + P, n_ud = s.n_ud;
        DevMem key, key_sorted, val;
        key.alloc(N * 4);
        key_sorted.alloc(N * 4);
        val.alloc(N * 4);
        m->m_ud_list_item.alloc(N * 4);
        m->m_ud_list_off.alloc((n_ud + 1) * 8);
        zeros(m->m_ud_pr_cnt, n_ud * 4, st);
        k_ud_list_keys<<<kGrid, kBlock, 0, st>>>(s, d_pu.as<int32_t>(), d_pi.as<int32_t>(), d_pd.as<int16_t>(), P,
                                                 key.as<uint32_t>(), val.as<uint32_t>(), m->m_ud_pr_cnt.as<uint32_t>());
        TSVD_CUDA(cudaGetLastError());
        sort_pairs(tmp, key.as<uint32_t>(), key_sorted.as<uint32_t>(), val.as<uint32_t>(),
                   m->m_ud_list_item.as<uint32_t>(), N, bits_for(n_ud), st);
        k_lower_bound_u32<<<ceil_div(n_ud + 1, kBlock), kBlock, 0, st>>>(key_sorted.as<uint32_t>(), N, n_ud,
                                                                         m->m_ud_list_off.as<uint64_t>());
        TSVD_CUDA(cudaGetLastError());
        s.ud_list_off = m->m_ud_list_off.as<uint64_t>();
        s.ud_list_item = m->m_ud_list_item.as<uint32_t>();
        s.ud_pr_cnt = m->m_ud_pr_cnt.as<uint32_t>();
        TSVD_CUDA(cudaStreamSynchronize(st));
    }

    // ---- pr items grouped by user, pr order kept (probe_items_by_user) ------
    {
        DevMem idx, idx_sorted, ukey, ukey_sorted;
        m->m_pr_item.alloc(P * 4);
        if (P) {
            idx.alloc(P * 4);
            idx_sorted.alloc(P * 4);
            ukey.alloc(P * 4);
            ukey_sorted.alloc(P * 4);
            k_iota<<<kGrid, kBlock, 0, st>>>(idx.as<uint32_t>(), P);
            TSVD_CUDA(cudaMemcpyAsync(ukey.p, d_pu.p, P * 4, cudaMemcpyDeviceToDevice, st));
            sort_pairs(tmp, ukey.as<uint32_t>(), ukey_sorted.as<uint32_t>(), idx.as<uint32_t>(),
                       idx_sorted.as<uint32_t>(), P, bits_for(U), st);
            k_gather_u32<<<kGrid, kBlock, 0, st>>>(d_pi.as<int32_t>(), idx_sorted.as<uint32_t>(), P,
                                                   m->m_pr_item.as<uint32_t>());
            TSVD_CUDA(cudaGetLastError());
        }
        std::vector<uint64_t> poff(U + 1, 0);
        for (uint32_t u = 0; u < U; ++u) poff[u + 1] = poff[u] + (uint64_t)pr.user_cnts[u];
        upload(m->m_pr_off, poff.data(), U + 1, st);
        s.pr_item = m->m_pr_item.as<uint32_t>();
        s.pr_off = m->m_pr_off.as<uint64_t>();
        TSVD_CUDA(cudaStreamSynchronize(st));
    }

    // ---- by-item index (ByItemIndex, src/tsvdx4p.rs:29-57) -------------------
    {
        DevMem idx, idx_sorted, ikey, ikey_sorted;
        idx.alloc(R * 4);
        idx_sorted.alloc(R * 4);
        ikey.alloc(R * 4);
        ikey_sorted.alloc(R * 4);
        k_iota<<<kGrid, kBlock, 0, st>>>(idx.as<uint32_t>(), R);
        TSVD_CUDA(cudaMemcpyAsync(ikey.p, d_ti.p, R * 4, cudaMemcpyDeviceToDevice, st));
        sort_pairs(tmp, ikey.as<uint32_t>(), ikey_sorted.as<uint32_t>(), idx.as<uint32_t>(), idx_sorted.as<uint32_t>(),
                   R, bits_for(I), st);
        m->m_irec.alloc(R * sizeof(Rec));
        k_item_records<<<kGrid, kBlock, 0, st>>>(m->m_rec.as<Rec>(), d_tu.as<int32_t>(), idx_sorted.as<uint32_t>(), R,
                                                 m->m_irec.as<Rec>());
        TSVD_CUDA(cudaGetLastError());
        // item offsets from the sorted item keys, on the device
        m->m_item_off.alloc((size_t)(I + 1) * 8);
        k_item_offsets<<<kGrid, kBlock, 0, st>>>(ikey_sorted.as<uint32_t>(), R, I, m->m_item_off.as<uint64_t>());
        TSVD_CUDA(cudaGetLastError());
        std::vector<uint64_t> ioff(I + 1, 0);
        TSVD_CUDA(cudaMemcpyAsync(ioff.data(), m->m_item_off.p, (size_t)(I + 1) * 8, cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaStreamSynchronize(st));
        std::vector<uint64_t> icnt(I, 0);
        for (uint32_t i = 0; i < I; ++i) icnt[i] = ioff[i + 1] - ioff[i];
        m->h_item_off = ioff;
        s.irec = m->m_irec.as<Rec>();
        s.item_off = m->m_item_off.as<uint64_t>();
        // work lists: heaviest first (longest-processing-time order)
        const std::vector<uint32_t> iw = heaviest_first(icnt.data(), I);
        upload(m->m_item_work, iw.data(), I, st);
        const std::vector<uint32_t> uw = heaviest_first(tr.user_cnts, U);
        upload(m->m_user_work, uw.data(), U, st);
        s.item_work = m->m_item_work.as<uint32_t>();
        s.n_item_work = I;
        s.user_work = m->m_user_work.as<uint32_t>();
        // fixed chunks of kChunkUsers ratings per item (deterministic split sums)
        std::vector<uint64_t> clo;
        std::vector<uint32_t> c0(I + 1, 0);
        for (uint32_t i = 0; i < I; ++i) {
            c0[i] = (uint32_t)clo.size();
            for (uint64_t a = ioff[i]; a < ioff[i + 1]; a += kChunkUsers) clo.push_back(a);
        }
        c0[I] = (uint32_t)clo.size();
        s.n_chunks = (uint32_t)clo.size();
        clo.push_back(R);
        upload(m->m_chunk_lo, clo.data(), clo.size(), st);
        upload(m->m_item_chunk0, c0.data(), c0.size(), st);
        s.chunk_lo = m->m_chunk_lo.as<uint64_t>();
        s.item_chunk0 = m->m_item_chunk0.as<uint32_t>();
        TSVD_CUDA(cudaStreamSynchronize(st));
    }
    setup_params(m);
}

// Per-model parameter tables and scratch (TxModel::new field order,
// src/tx.rs:600-648). The dataset part of m->d (sizes, records, indices) must
// already be set; models of one group share it and differ only here.
void setup_params(tsvd_model* m) {
    const tsvd_config& c = m->cfg;
    cudaStream_t st = m->stream;
    DeviceState& s = m->d;
    const uint32_t U = s.n_users, I = s.n_items, F = s.F, Fs = s.Fs;
    m->m_chunk_part.alloc((size_t)s.n_chunks * Fs * 4);
    m->m_chunk_epart.alloc((size_t)s.n_chunks * 4);
    s.chunk_part = m->m_chunk_part.as<float>();
    s.chunk_epart = m->m_chunk_epart.as<float>();
    {
        const size_t NF = c.n_freq_bins, T = c.n_time_bins;
        // rand_array2 draws, in TxModel::new order, from one seeded stream:
        // ufeat, ifeat, yfeat, yfeat_day (low_memory = false only), then
        // (after the zero tables) ifeat_freq
        m->m_ufeat.alloc((size_t)U * Fs * 4);
        m->m_ifeat.alloc((size_t)I * Fs * 4);
        m->m_yfeat.alloc((size_t)I * Fs * 4);
        m->m_ifeat_freq.alloc((size_t)I * NF * Fs * 4);
        std::vector<NormalTable> drawn = {{m->m_ufeat.as<float>(), U, F, Fs, c.sigma_u},
                                          {m->m_ifeat.as<float>(), I, F, Fs, c.sigma_i},
                                          {m->m_yfeat.as<float>(), I, F, Fs, c.sigma_y}};
        if (!c.low_memory) {
            m->m_yfeat_day.alloc((size_t)I * Fs * 4);
            drawn.push_back({m->m_yfeat_day.as<float>(), I, F, Fs, c.sigma_yd});
            zeros(m->m_ufeat_day, (size_t)s.n_ud * Fs * 4, st);
            zeros(m->m_ycache_day, (size_t)s.n_ud * Fs * 4, st);
            zeros(m->m_dyd_fix, (size_t)I * Fs * 8, st);
        }
        drawn.push_back({m->m_ifeat_freq.as<float>(), (uint64_t)I * NF, F, Fs, c.sigma_iqf});
        if (F > 0) {
            device_normal_tables(drawn.data(), (int)drawn.size(), c.seed, st);
        } else {
            // n_feat = 0 draws nothing (rand_array2 of an [n, 0] array)
            for (const NormalTable& t : drawn)
                TSVD_CUDA(cudaMemsetAsync(t.dst, 0, t.rows * t.stride * sizeof(float), st));
        }
        zeros(m->m_ufeat2, (size_t)U * Fs * 4, st);
        zeros(m->m_ycache, (size_t)U * Fs * 4, st);
        zeros(m->m_alpha_u, U * 4, st);
        zeros(m->m_but_bin, (size_t)U * T * 4, st);
        zeros(m->m_bit_bin, (size_t)I * T * 4, st);
        zeros(m->m_ybias, I * 4, st);
        zeros(m->m_ycache_bias, U * 4, st);
        zeros(m->m_ubias_day, s.n_ud * 4, st);
        zeros(m->m_ibias_freq, (size_t)I * NF * 4, st);
        zeros(m->m_ubias, U * 4, st);
        zeros(m->m_ibias, I * 4, st);
        m->m_cu.alloc(U * 4);
        k_fill<<<kGrid, kBlock, 0, st>>>(m->m_cu.as<float>(), U, 1.0f);
        TSVD_CUDA(cudaGetLastError());
        zeros(m->m_cut, s.n_ud * 4, st);
        zeros(m->m_thresholds, 16, st);
        zeros(m->m_g_user, (size_t)U * Fs * 4, st);
        if (c.low_memory) zeros(m->m_qe0, (size_t)I * Fs * 4, st);
        zeros(m->m_e_user, U * 4, st);
        zeros(m->m_counters, 64, st);
        m->m_perm.alloc(U * 4);
        if (m->opts.precision >= TSVD_PREC_BF16_READ) {
            m->m_bf_ifeat.alloc((size_t)I * Fs * 2);
            m->m_bf_qf0.alloc((size_t)I * Fs * 2);
            m->m_bf_yfeat.alloc((size_t)I * Fs * 2);
        }
        if (m->opts.precision >= TSVD_PREC_BF16_READ_ALL) {
            m->m_bf_pyc.alloc((size_t)U * Fs * 2);
            m->m_bf_ufeat2.alloc((size_t)U * Fs * 2);
        }
        s.ubias = m->m_ubias.as<float>(); s.ibias = m->m_ibias.as<float>();
        s.ufeat = m->m_ufeat.as<float>(); s.ufeat2 = m->m_ufeat2.as<float>();
        s.ifeat = m->m_ifeat.as<float>(); s.yfeat = m->m_yfeat.as<float>();
        s.ycache = m->m_ycache.as<float>();
        s.yfeat_day = c.low_memory ? nullptr : m->m_yfeat_day.as<float>();
        s.alpha_u = m->m_alpha_u.as<float>(); s.but_bin = m->m_but_bin.as<float>();
        s.bit_bin = m->m_bit_bin.as<float>(); s.ybias = m->m_ybias.as<float>();
        s.ycache_bias = m->m_ycache_bias.as<float>(); s.ubias_day = m->m_ubias_day.as<float>();
        s.ufeat_day = c.low_memory ? nullptr : m->m_ufeat_day.as<float>();
        s.ycache_day = c.low_memory ? nullptr : m->m_ycache_day.as<float>();
        s.dyd_fix = c.low_memory ? nullptr : m->m_dyd_fix.as<unsigned long long>();
        s.qe0 = c.low_memory ? m->m_qe0.as<float>() : nullptr;
        s.ibias_freq = m->m_ibias_freq.as<float>(); s.ifeat_freq = m->m_ifeat_freq.as<float>();
        s.cu = m->m_cu.as<float>(); s.cut = m->m_cut.as<float>();
        s.thresholds = m->m_thresholds.as<float>();
        s.g_user = m->m_g_user.as<float>(); s.e_user = m->m_e_user.as<float>();
        s.pyc = s.g_user;
        s.counters = m->m_counters.as<uint32_t>();
        if (c.has_ordinal_head) {
            TSVD_CUDA(cudaMemcpyAsync(m->m_thresholds.p, c.ordinal_head.th_init, 16, cudaMemcpyHostToDevice, st));
            std::memcpy(m->h_thresholds, c.ordinal_head.th_init, 16);
        }
    }
    TSVD_CUDA(cudaStreamSynchronize(st));
    m->ycache_valid = false;  // ycache starts at zero, as in the reference
}

}  // namespace tsvd
