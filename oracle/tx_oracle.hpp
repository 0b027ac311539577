// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the tsvdx4 path. Only the
// test suite, the smoke check and bench.py's CPU-baseline leg load it, as the
// checker; the CUDA library never includes, links or calls it.
//
// A restatement, in the reference's operation order, of
//   src/tx.rs        TxModel in tx4 mode (neighbourhood off):
//                    SparseUD :21-84, freq_bin :87-90, day_ranges :93-105,
//                    time_bin/dev :285-300, factor_parts :303-339,
//                    rebuild_ycache(_day) :391-454, new :460-649,
//                    predict_subscores :651-711, predict :713-724,
//                    fit_epoch :734-1115
//   src/lib.rs       calc_gbias :463-467, calc_user_offsets :470-483,
//                    get_users :486-494, rand_array2 :64-67,
//                    OrdinalHead :500-609, calc_rmse :659-672,
//                    gen_preds :689-700
//   src/tsvdx4p.rs   Tsvdx4pModel: apply_nsvd_deltas :341-385,
//                    fit_epoch_user :390-639, fit_epoch_item :644-762,
//                    fit_epoch :798-805
// The scalar type is a template parameter: float reproduces the reference's
// f32 arithmetic (build with -ffp-contract=off, no fast-math), double is the
// FP64 twin used to state the error of reduced-precision forms.
#pragma once
#include <algorithm>
#include <atomic>
#include <math.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "rand09.hpp"

namespace oracle {

struct OrdinalCfg {
    float th_init[4];
    float th_gap;
    float lr_t;
    float reg_t;
};

// Field-for-field mirror of TxConfig (src/tx.rs:128-204).
struct Config {
    uint64_t n_feat, n_epochs, seed;
    bool shuffle_users;
    uint64_t n_time_bins;
    float beta;
    uint64_t n_freq_bins;
    float lr_u, lr_ud, lr_u2, lr_ub, lr_ubd, lr_i, lr_ib, lr_y, lr_yb, lr_yd, lr_tu, lr_ti, lr_ta, lr_ibf, lr_iqf,
        lr_cu;
    float reg_iqf, reg_cu, reg_u, reg_u2, reg_ud, reg_i, reg_y, reg_yd;
    float sigma_iqf, sigma_u, sigma_i, sigma_y, sigma_yd;
    uint64_t reset_u_epoch;
    uint64_t max_neighbors;
    float lr_w, lr_c, reg_w, reg_c, lr_w_day, lr_c_day, reg_w_day, reg_c_day;
    float w_bias, w_factor, w_nbr;
    bool sum_err_bug;
    float lambda1, lambda2;
    bool has_ordinal;
    OrdinalCfg ordinal;
    bool save_ifeat, low_memory, full_su;
};

// Borrowed view of a Dataset (src/lib.rs:227-242); residuals/raw_ratings are
// null for a MaskedDataset (src/lib.rs:421-455).
struct DataView {
    const int32_t* user_idxs;
    const int32_t* user_cnts;
    const int32_t* item_idxs;
    const int8_t* raw_ratings;
    const float* residuals;
    const int16_t* dates;
    const int8_t* is_test;
    size_t n_users, n_items, n_ratings;
};

inline float sigmoidf(float x) { return 1.0f / (1.0f + ::expf(-x)); }

// src/lib.rs:500-609
struct OrdinalHead {
    OrdinalCfg cfg;
    float th[4];
    void enforce_sorted_with_gap() {
        std::sort(th, th + 4);
        for (int k = 1; k < 4; ++k) {
            float min_ok = th[k - 1] + cfg.th_gap;
            if (th[k] < min_ok) th[k] = min_ok;
        }
    }
    void predict_probs(float score, float p[5]) const {
        float f[6];
        f[0] = 0.0f;
        f[5] = 1.0f;
        for (int k = 1; k < 5; ++k) f[k] = sigmoidf(th[k - 1] - score);
        for (int k = 0; k < 5; ++k) p[k] = f[k + 1] - f[k];
    }
    float grad(float score, int y, float g_t[4]) const {
        float f[6], a[6];
        f[0] = 0.0f;
        f[5] = 1.0f;
        for (int k = 1; k < 5; ++k) f[k] = sigmoidf(th[k - 1] - score);
        for (int k = 0; k < 6; ++k) a[k] = f[k] * (1.0f - f[k]);
        if (y < 1 || y > 5) throw std::runtime_error("ordinal head: rating outside 1..5");
        float p_y = ::fmaxf(f[y] - f[y - 1], 1e-6f);
        float g_ds = (a[y] - a[y - 1]) / p_y;
        for (int k = 0; k < 4; ++k) g_t[k] = 0.0f;
        if (y >= 2) g_t[y - 2] += a[y - 1] / p_y;
        if (y <= 4) g_t[y - 1] -= a[y] / p_y;
        return g_ds;
    }
    void update(const float g_t[4]) {
        for (int k = 0; k < 4; ++k) {
            float tk = th[k];
            th[k] -= cfg.lr_t * (g_t[k] + cfg.reg_t * tk);
        }
    }
};

inline size_t freq_bin(uint32_t day_cnt, size_t n_freq_bins) {
    if (day_cnt <= 1) return 0;
    float v = ::floorf(::log2f((float)day_cnt));
    float cap = (float)(n_freq_bins - 1);
    return (size_t)::fminf(v, cap);
}

inline double calc_gbias(const DataView& tr) {
    double s = 0.0;
    for (size_t t = 0; t < tr.n_ratings; ++t) s += (double)tr.residuals[t];
    return (float)(s / (double)tr.n_ratings);
}

inline std::vector<size_t> calc_user_offsets(const DataView& tr) {
    for (size_t t = 1; t < tr.n_ratings; ++t)
        if (tr.user_idxs[t] < tr.user_idxs[t - 1])
            throw std::runtime_error("dataset is not user-sorted at index " + std::to_string(t));
    std::vector<size_t> off(tr.n_users + 1, 0);
    for (size_t u = 0; u < tr.n_users; ++u) off[u + 1] = off[u] + (size_t)tr.user_cnts[u];
    return off;
}

inline std::vector<uint32_t> get_users(size_t n, bool shuffle_users, uint64_t seed, uint64_t epoch) {
    std::vector<uint32_t> users(n);
    for (size_t u = 0; u < n; ++u) users[u] = (uint32_t)u;
    if (shuffle_users) {
        StdRng rng = StdRng::seed_from_u64(seed ^ (epoch * 0x9E3779B97F4A7C15ull));
        shuffle(users, rng);
    }
    return users;
}

// SparseUD (src/tx.rs:21-84): per-user sorted distinct days over train + pr.
struct SparseUD {
    std::vector<size_t> starts;
    std::vector<int16_t> dates;
    std::vector<uint32_t> day_cnts;
    SparseUD() = default;
    SparseUD(const DataView& a, const DataView& b) {
        std::vector<std::vector<int16_t>> per(a.n_users);
        for (size_t t = 0; t < a.n_ratings; ++t) per[a.user_idxs[t]].push_back(a.dates[t]);
        for (size_t t = 0; t < b.n_ratings; ++t) per[b.user_idxs[t]].push_back(b.dates[t]);
        starts.reserve(a.n_users + 1);
        for (size_t u = 0; u < a.n_users; ++u) {
            starts.push_back(dates.size());
            auto& s = per[u];
            std::sort(s.begin(), s.end());
            if (s.empty()) continue;
            int16_t prev = s[0];
            uint32_t cnt = 1;
            for (size_t k = 1; k < s.size(); ++k) {
                if (s[k] == prev) {
                    ++cnt;
                } else {
                    dates.push_back(prev);
                    day_cnts.push_back(cnt);
                    prev = s[k];
                    cnt = 1;
                }
            }
            dates.push_back(prev);
            day_cnts.push_back(cnt);
        }
        starts.push_back(dates.size());
    }
    size_t n_total() const { return dates.size(); }
    // -1 when (u, day) is absent.
    long index(size_t u, int16_t day) const {
        auto b = dates.begin() + starts[u], e = dates.begin() + starts[u + 1];
        auto it = std::lower_bound(b, e, day);
        if (it == e || *it != day) return -1;
        return (long)(it - dates.begin());
    }
};

inline std::vector<std::pair<size_t, size_t>> day_ranges(const int16_t* dates, size_t start, size_t end) {
    std::vector<std::pair<size_t, size_t>> r;
    if (start == end) return r;
    size_t rs = start;
    for (size_t i = start + 1; i < end; ++i)
        if (dates[i] != dates[i - 1]) {
            r.push_back({rs, i - 1});
            rs = i;
        }
    r.push_back({rs, end - 1});
    return r;
}

template <class T>
struct Mat {
    size_t rows = 0, cols = 0;
    std::vector<T> v;
    Mat() = default;
    Mat(size_t r, size_t c) : rows(r), cols(c), v(r * c, T(0)) {}
    T* row(size_t r) { return v.data() + r * cols; }
    const T* row(size_t r) const { return v.data() + r * cols; }
    T& at(size_t r, size_t c) { return v[r * cols + c]; }
    const T& at(size_t r, size_t c) const { return v[r * cols + c]; }
    void fill(T x) { std::fill(v.begin(), v.end(), x); }
};

inline double powT(double a, double b) { return ::pow(a, b); }
inline float powT(float a, float b) { return ::powf(a, b); }
inline double sqrtT(double a) { return ::sqrt(a); }
inline float sqrtT(float a) { return ::sqrtf(a); }
inline double absT(double a) { return ::fabs(a); }
inline float absT(float a) { return ::fabsf(a); }

template <class T>
Mat<T> rand_array2(size_t rows, size_t cols, StdRng& rng, float sigma) {
    Mat<T> m(rows, cols);
    for (size_t k = 0; k < rows * cols; ++k) m.v[k] = (T)normal_f32(rng, sigma);
    return m;
}

// TxModel (src/tx.rs:210-272) in tx4 mode.
template <class T>
struct TxModel {
    Config cfg;
    T gbias;
    std::vector<T> ubias, ibias;
    Mat<T> ufeat, ufeat2, ifeat, yfeat, ycache, yfeat_day;
    int32_t day_range = 0;
    std::vector<T> tu_mean, alpha_u;
    Mat<T> but_bin, bit_bin;
    std::vector<T> ybias, ycache_bias;
    SparseUD ud;
    std::vector<T> ubias_day;
    Mat<T> ufeat_day, ycache_day;
    Mat<T> ibias_freq, ifeat_freq;
    std::vector<T> cu, cut;
    bool has_ordinal = false;
    OrdinalHead ordinal;
    size_t n_users = 0, n_items = 0;
    std::vector<size_t> user_offsets;
    std::vector<std::vector<uint32_t>> probe_items_by_user, probe_items_by_ud;
    // Optional injected per-epoch user orders (epoch -> permutation).
    std::vector<std::vector<uint32_t>> injected_order;

    TxModel(const DataView& tr, const DataView& pr, const Config& c) : cfg(c) {
        if (c.lr_w != 0 || c.lr_c != 0 || c.lr_w_day != 0 || c.lr_c_day != 0)
            throw std::runtime_error("neighbourhood terms (tx5/tx6) are outside the tsvdx4 path");
        StdRng rng = StdRng::seed_from_u64(c.seed);
        n_users = tr.n_users;
        n_items = tr.n_items;
        const size_t F = c.n_feat;
        std::vector<float> tum(n_users, 0.0f);
        int32_t dr = 0;
        for (size_t t = 0; t < tr.n_ratings; ++t) {
            tum[tr.user_idxs[t]] += (float)tr.dates[t];
            dr = std::max(dr, (int32_t)tr.dates[t] + 1);
        }
        for (size_t u = 0; u < n_users; ++u)
            if (tr.user_cnts[u] > 0) tum[u] /= (float)tr.user_cnts[u];
        day_range = dr;
        tu_mean.assign(tum.begin(), tum.end());
        ud = SparseUD(tr, pr);
        const size_t n_ud = ud.n_total();
        user_offsets = calc_user_offsets(tr);
        gbias = (T)calc_gbias(tr);
        probe_items_by_user.assign(n_users, {});
        probe_items_by_ud.assign(n_ud, {});
        if (c.full_su) {
            for (size_t t = 0; t < pr.n_ratings; ++t) {
                size_t u = pr.user_idxs[t];
                uint32_t item = (uint32_t)pr.item_idxs[t];
                probe_items_by_user[u].push_back(item);
                long idx = ud.index(u, pr.dates[t]);
                if (idx >= 0) probe_items_by_ud[idx].push_back(item);
            }
        }
        ubias.assign(n_users, T(0));
        ibias.assign(n_items, T(0));
        ufeat = rand_array2<T>(n_users, F, rng, c.sigma_u);
        ufeat2 = Mat<T>(n_users, F);
        ifeat = rand_array2<T>(n_items, F, rng, c.sigma_i);
        yfeat = rand_array2<T>(n_items, F, rng, c.sigma_y);
        ycache = Mat<T>(n_users, F);
        yfeat_day = c.low_memory ? Mat<T>(0, F) : rand_array2<T>(n_items, F, rng, c.sigma_yd);
        alpha_u.assign(n_users, T(0));
        but_bin = Mat<T>(n_users, c.n_time_bins);
        bit_bin = Mat<T>(n_items, c.n_time_bins);
        ybias.assign(n_items, T(0));
        ycache_bias.assign(n_users, T(0));
        ubias_day.assign(n_ud, T(0));
        ufeat_day = c.low_memory ? Mat<T>(0, F) : Mat<T>(n_ud, F);
        ycache_day = c.low_memory ? Mat<T>(0, F) : Mat<T>(n_ud, F);
        ibias_freq = Mat<T>(n_items, c.n_freq_bins);
        ifeat_freq = rand_array2<T>(n_items * c.n_freq_bins, F, rng, c.sigma_iqf);
        cu.assign(n_users, T(1));
        cut.assign(n_ud, T(0));
        has_ordinal = c.has_ordinal;
        if (has_ordinal) {
            ordinal.cfg = c.ordinal;
            std::memcpy(ordinal.th, c.ordinal.th_init, sizeof(ordinal.th));
        }
    }

    size_t time_bin(int32_t day) const {
        int64_t num = (int64_t)day * (int64_t)cfg.n_time_bins;
        size_t b = (size_t)(num / (int64_t)day_range);
        return std::min(b, (size_t)cfg.n_time_bins - 1);
    }
    T dev(size_t u, int32_t day) const {
        T dt = (T)day - tu_mean[u];
        if (dt == T(0)) return T(0);
        T s = dt > T(0) ? T(1) : T(-1);
        return s * powT(absT(dt), (T)cfg.beta);
    }

    // (bias part, dot part) -- src/tx.rs:303-339
    void factor_parts(size_t u, size_t i, int32_t day, T& bias_part, T& dot_part) const {
        const size_t F = cfg.n_feat, NF = cfg.n_freq_bins;
        size_t b = time_bin(day);
        T dv = dev(u, day);
        long idx = ud.index(u, (int16_t)day);
        size_t f = idx >= 0 ? freq_bin(ud.day_cnts[idx], NF) : 0;
        T bu_day = idx >= 0 ? ubias_day[idx] : T(0);
        T bu_t = ubias[u] + but_bin.at(u, b) + alpha_u[u] * dv + bu_day + ycache_bias[u];
        T bi_t = ibias[i] + bit_bin.at(i, b) + ibias_freq.at(i, f);
        T cu_t = cu[u] + (idx >= 0 ? cut[idx] : T(0));
        const T *pu = ufeat.row(u), *pu2 = ufeat2.row(u), *su = ycache.row(u);
        const T *qi = ifeat.row(i), *qf = ifeat_freq.row(i * NF + f);
        T dot = T(0);
        for (size_t k = 0; k < F; ++k) {
            T qe = qi[k] + qf[k];
            T pe = pu[k] + su[k] + dv * pu2[k];
            if (!cfg.low_memory && idx >= 0) {
                pe += ufeat_day.at(idx, k);
                pe += ycache_day.at(idx, k);
            }
            dot += pe * qe;
        }
        bias_part = gbias + bu_t + bi_t * cu_t;
        dot_part = dot;
    }

    // src/tx.rs:713-724
    T predict(size_t u, size_t i, int32_t day) const {
        T bp, dp;
        factor_parts(u, i, day, bp, dp);
        T score = bp + dp + T(0);
        if (has_ordinal) {
            float p[5];
            ordinal.predict_probs((float)score, p);
            return (T)(1.0f * p[0] + 2.0f * p[1] + 3.0f * p[2] + 4.0f * p[3] + 5.0f * p[4]);
        }
        return score;
    }

    // src/tx.rs:663-711 -> [bias, mf, nsvd1]
    void predict_subscores(size_t u, size_t i, int32_t day, T out[3]) const {
        const size_t F = cfg.n_feat, NF = cfg.n_freq_bins;
        size_t b = time_bin(day);
        T dv = dev(u, day);
        long idx = ud.index(u, (int16_t)day);
        size_t f = idx >= 0 ? freq_bin(ud.day_cnts[idx], NF) : 0;
        T bu_day = idx >= 0 ? ubias_day[idx] : T(0);
        T bi_t = ibias[i] + bit_bin.at(i, b) + ibias_freq.at(i, f);
        T cu_t = cu[u] + (idx >= 0 ? cut[idx] : T(0));
        T bias = gbias + ubias[u] + ibias[i] + ibias_freq.at(i, f) + but_bin.at(u, b) + alpha_u[u] * dv + bu_day +
                 bit_bin.at(i, b) + bi_t * (cu_t - T(1)) + ycache_bias[u];
        const T *pu = ufeat.row(u), *pu2 = ufeat2.row(u), *su = ycache.row(u);
        const T *qi = ifeat.row(i), *qf = ifeat_freq.row(i * NF + f);
        T mf = T(0), ns = T(0);
        for (size_t k = 0; k < F; ++k) {
            T qe = qi[k] + qf[k];
            T pe = pu[k] + dv * pu2[k];
            if (!cfg.low_memory && idx >= 0) pe += ufeat_day.at(idx, k);
            mf += pe * qe;
            T se = su[k];
            if (!cfg.low_memory && idx >= 0) se += ycache_day.at(idx, k);
            ns += se * qe;
        }
        out[0] = bias;
        out[1] = mf;
        out[2] = ns;
    }

    // src/tx.rs:391-418
    void rebuild_ycache(const DataView& tr, const DataView& pr) {
        const size_t F = cfg.n_feat;
        ycache.fill(T(0));
        std::fill(ycache_bias.begin(), ycache_bias.end(), T(0));
        auto add = [&](const DataView& d) {
            for (size_t t = 0; t < d.n_ratings; ++t) {
                size_t u = d.user_idxs[t], i = d.item_idxs[t];
                T* su = ycache.row(u);
                const T* y = yfeat.row(i);
                for (size_t k = 0; k < F; ++k) su[k] += y[k];
                ycache_bias[u] += ybias[i];
            }
        };
        add(tr);
        add(pr);
        for (size_t u = 0; u < n_users; ++u) {
            int32_t cnt = tr.user_cnts[u] + pr.user_cnts[u];
            if (cnt > 0) {
                T* su = ycache.row(u);
                T nrm = sqrtT((T)(float)cnt);
                for (size_t k = 0; k < F; ++k) su[k] /= nrm;
                ycache_bias[u] /= nrm;
            }
        }
    }

    // src/tx.rs:420-454
    void rebuild_ycache_day(const DataView& tr, const DataView& pr) {
        const size_t F = cfg.n_feat;
        ycache_day.fill(T(0));
        std::vector<float> cnts(ud.n_total(), 0.0f);
        auto add = [&](const DataView& d) {
            for (size_t t = 0; t < d.n_ratings; ++t) {
                long idx = ud.index(d.user_idxs[t], d.dates[t]);
                if (idx < 0) continue;
                cnts[idx] += 1.0f;
                T* row = ycache_day.row(idx);
                const T* y = yfeat_day.row(d.item_idxs[t]);
                for (size_t k = 0; k < F; ++k) row[k] += y[k];
            }
        };
        add(pr);
        add(tr);
        for (size_t idx = 0; idx < ud.n_total(); ++idx)
            if (cnts[idx] > 0.0f) {
                T nrm = sqrtT((T)cnts[idx]);
                T* row = ycache_day.row(idx);
                for (size_t k = 0; k < F; ++k) row[k] /= nrm;
            }
    }

    std::vector<uint32_t> users_for_epoch(uint64_t epoch) const {
        if (epoch < injected_order.size() && !injected_order[epoch].empty()) return injected_order[epoch];
        return get_users(n_users, cfg.shuffle_users, cfg.seed, epoch);
    }

    // src/tx.rs:734-1115 (tx4 mode)
    void fit_epoch(const DataView& tr, const DataView& pr, uint64_t epoch) {
        const Config c = cfg;
        const size_t F = c.n_feat, NF = c.n_freq_bins;
        const bool use_probe = c.full_su, low_mem = c.low_memory;
        if (epoch == c.reset_u_epoch) {
            ufeat.fill(T(0));
            ufeat2.fill(T(0));
        }
        std::vector<uint32_t> users = users_for_epoch(epoch);
        std::vector<T> su(F), sum_err_q(F), sum_err_q_day(low_mem ? 0 : F), su_day(low_mem ? 0 : F), su_freq(F);
        for (uint32_t uu : users) {
            const size_t u = uu;
            const size_t start = user_offsets[u], end = user_offsets[u + 1];
            const size_t cnt = end - start;
            if (cnt == 0) continue;
            std::vector<std::pair<size_t, size_t>> drs;
            if (!low_mem) drs = day_ranges(tr.dates, start, end);
            std::fill(su.begin(), su.end(), T(0));
            T su_bias = T(0);
            for (size_t t = start; t < end; ++t) {
                size_t j = tr.item_idxs[t];
                const T* y = yfeat.row(j);
                for (size_t k = 0; k < F; ++k) su[k] += y[k];
                su_bias += ybias[j];
            }
            size_t total_cnt = cnt;
            if (use_probe) {
                for (uint32_t j : probe_items_by_user[u]) {
                    const T* y = yfeat.row(j);
                    for (size_t k = 0; k < F; ++k) su[k] += y[k];
                    su_bias += ybias[j];
                }
                total_cnt = cnt + probe_items_by_user[u].size();
            }
            const T norm = sqrtT((T)(float)total_cnt);
            for (size_t k = 0; k < F; ++k) su[k] /= norm;
            std::copy(su.begin(), su.end(), ycache.row(u));
            su_bias /= norm;
            ycache_bias[u] = su_bias;

            std::fill(sum_err_q.begin(), sum_err_q.end(), T(0));
            if (!low_mem) std::fill(sum_err_q_day.begin(), sum_err_q_day.end(), T(0));
            T sum_err = T(0);
            if (!low_mem) std::fill(su_day.begin(), su_day.end(), T(0));
            std::fill(su_freq.begin(), su_freq.end(), T(0));
            T norm_day = T(0);
            size_t dr_idx = 0, cur_freq_bin = 0;

            for (size_t t = start; t < end; ++t) {
                const size_t i = tr.item_idxs[t];
                const T r = (T)tr.residuals[t];
                const int32_t day = tr.dates[t];
                const int16_t day16 = tr.dates[t];
                const size_t b = time_bin(day);
                const T dv = dev(u, day);
                size_t day_start = 0, day_stop = 0;
                if (!low_mem) {
                    day_start = drs[dr_idx].first;
                    day_stop = drs[dr_idx].second;
                }
                if (!low_mem && t == day_start) {
                    std::fill(sum_err_q_day.begin(), sum_err_q_day.end(), T(0));
                    std::fill(su_day.begin(), su_day.end(), T(0));
                    std::fill(su_freq.begin(), su_freq.end(), T(0));
                    long idx_day = ud.index(u, day16);
                    cur_freq_bin = idx_day >= 0 ? freq_bin(ud.day_cnts[idx_day], NF) : 0;
                    for (size_t td = day_start; td <= day_stop; ++td) {
                        const T* y = yfeat_day.row(tr.item_idxs[td]);
                        for (size_t k = 0; k < F; ++k) su_day[k] += y[k];
                    }
                    float day_cnt = (float)(day_stop - day_start + 1);
                    if (use_probe && idx_day >= 0) {
                        for (uint32_t j : probe_items_by_ud[idx_day]) {
                            const T* y = yfeat_day.row(j);
                            for (size_t k = 0; k < F; ++k) su_day[k] += y[k];
                            day_cnt += 1.0f;
                        }
                    }
                    norm_day = sqrtT((T)day_cnt);
                    for (size_t k = 0; k < F; ++k) su_day[k] /= norm_day;
                    for (size_t k = 0; k < F; ++k) su_freq[k] /= norm_day;
                }
                const size_t f = cur_freq_bin;

                const long idx = ud.index(u, day16);
                const T bu_day = idx >= 0 ? ubias_day[idx] : T(0);
                const T bu_t = ubias[u] + but_bin.at(u, b) + alpha_u[u] * dv + bu_day + ycache_bias[u];
                const T bi_t = ibias[i] + bit_bin.at(i, b) + ibias_freq.at(i, f);
                const T cu_t = cu[u] + (idx >= 0 ? cut[idx] : T(0));
                {
                    const T *pu = ufeat.row(u), *pu2 = ufeat2.row(u), *srow = ycache.row(u);
                    const T *qi = ifeat.row(i), *qf = ifeat_freq.row(i * NF + f);
                    T dot = T(0);
                    for (size_t k = 0; k < F; ++k) {
                        T qe = qi[k] + qf[k];
                        T pe = pu[k] + srow[k] + dv * pu2[k];
                        if (!low_mem) {
                            if (idx >= 0) pe += ufeat_day.at(idx, k);
                            pe += su_day[k] + su_freq[k];
                        }
                        dot += pe * qe;
                    }
                    const T bias_part = gbias + bu_t + bi_t * cu_t;
                    const T score = bias_part + dot + T(0);
                    T err;
                    if (has_ordinal) {
                        float g_t[4];
                        err = (T)ordinal.grad((float)score, (int)tr.raw_ratings[t], g_t);
                        ordinal.update(g_t);
                    } else {
                        err = score - r;
                    }
                    const T err_b = err * (T)c.w_bias, err_d = err * (T)c.w_factor;

                    ubias[u] -= (T)c.lr_ub * err_b;
                    but_bin.at(u, b) -= (T)c.lr_tu * err_b;
                    alpha_u[u] -= (T)c.lr_ta * err_b * dv;
                    if (idx >= 0) ubias_day[idx] -= (T)c.lr_ubd * err_b;
                    ibias[i] -= (T)c.lr_ib * (err_b * cu_t);
                    bit_bin.at(i, b) -= (T)c.lr_ti * (err_b * cu_t);
                    ibias_freq.at(i, f) -= (T)c.lr_ibf * (err_b * cu_t);
                    cu[u] -= (T)c.lr_cu * (err_b * bi_t + (T)c.reg_cu * (cu[u] - T(1)));

                    const bool has_ud = !low_mem && c.lr_ud != 0.0f;
                    if (!c.sum_err_bug) sum_err += err_b;
                    T* qrow = ifeat.row(i);
                    T* qfrow = ifeat_freq.row(i * NF + f);
                    T* prow = ufeat.row(u);
                    T* p2row = ufeat2.row(u);
                    for (size_t k = 0; k < F; ++k) {
                        const T qi_k = qrow[k], qf_k = qfrow[k];
                        const T qe = qi_k + qf_k;
                        const T pu_k = prow[k], pu2_k = p2row[k];
                        sum_err_q[k] += err_d * qe;
                        if (!low_mem) sum_err_q_day[k] += err_d * qe;
                        if (c.sum_err_bug) sum_err += err_b;
                        prow[k] -= (T)c.lr_u * (err_d * qe + (T)c.reg_u * pu_k);
                        p2row[k] -= (T)c.lr_u2 * (err_d * qe * dv + (T)c.reg_u2 * pu2_k);
                        T pud_k = T(0);
                        if (has_ud && idx >= 0) {
                            T pud = ufeat_day.at(idx, k);
                            ufeat_day.at(idx, k) -= (T)c.lr_ud * (err_d * qe + (T)c.reg_ud * pud);
                            pud_k = pud;
                        }
                        const T pe = pu_k + dv * pu2_k + pud_k + su[k] + (low_mem ? T(0) : su_day[k] + su_freq[k]);
                        qrow[k] -= (T)c.lr_i * (err_d * pe + (T)c.reg_i * qi_k);
                        qfrow[k] -= (T)c.lr_iqf * (err_d * pe + (T)c.reg_iqf * qf_k);
                    }
                }
                if (!low_mem && t == day_stop) {
                    for (size_t td = day_start; td <= day_stop; ++td) {
                        T* y = yfeat_day.row(tr.item_idxs[td]);
                        for (size_t k = 0; k < F; ++k) {
                            T yj = y[k];
                            y[k] -= (T)c.lr_yd * (sum_err_q_day[k] / norm_day + (T)c.reg_yd * yj);
                        }
                    }
                    ++dr_idx;
                }
            }
            for (size_t t = start; t < end; ++t) {
                size_t j = tr.item_idxs[t];
                T* y = yfeat.row(j);
                for (size_t k = 0; k < F; ++k) {
                    T yj = y[k];
                    y[k] -= (T)c.lr_y * (sum_err_q[k] / norm + (T)c.reg_y * yj);
                }
                ybias[j] -= (T)c.lr_yb * (sum_err / norm);
            }
        }
        rebuild_ycache(tr, pr);
        if (!low_mem) rebuild_ycache_day(tr, pr);
        if (has_ordinal) ordinal.enforce_sorted_with_gap();
    }

    // ---------------- Tsvdx4pModel schedule (src/tsvdx4p.rs) ----------------
    struct ByItem {
        std::vector<size_t> starts;
        std::vector<uint32_t> user, rating;
    };
    ByItem by_item;
    void build_by_item(const DataView& tr) {
        std::vector<uint32_t> counts(n_items, 0);
        for (size_t t = 0; t < tr.n_ratings; ++t) counts[tr.item_idxs[t]]++;
        by_item.starts.assign(n_items + 1, 0);
        for (size_t i = 0; i < n_items; ++i) by_item.starts[i + 1] = by_item.starts[i] + counts[i];
        by_item.user.assign(tr.n_ratings, 0);
        by_item.rating.assign(tr.n_ratings, 0);
        std::vector<size_t> pos(by_item.starts.begin(), by_item.starts.end() - 1);
        for (size_t t = 0; t < tr.n_ratings; ++t) {
            size_t i = tr.item_idxs[t];
            by_item.user[pos[i]] = (uint32_t)tr.user_idxs[t];
            by_item.rating[pos[i]] = (uint32_t)t;
            pos[i]++;
        }
    }

    // The NSVD1 deltas of a set of users (one rayon chunk's NsvdDelta,
    // src/tsvdx4p.rs:63-80).
    struct PDeltas {
        Mat<T> dy, dyd;
        std::vector<T> dyb;
        std::vector<uint32_t> nc;
        PDeltas(size_t I, size_t F, bool day) : dy(I, F), dyd(day ? I : 0, F), dyb(I, T(0)), nc(I, 0) {}
    };

    // src/tsvdx4p.rs:390-639 followed by :341-385 and the cache rebuild.
    void fit_epoch_user_p(const DataView& tr, const DataView& pr, uint64_t epoch, float nsvd_norm_exp,
                          size_t n_threads) {
        const Config c = cfg;
        const size_t F = c.n_feat;
        const bool low_mem = c.low_memory;
        user_phase_prologue_p(epoch);
        std::vector<uint32_t> users = users_for_epoch(epoch);
        n_threads = std::max<size_t>(n_threads, 1);
        size_t chunk = std::max<size_t>((users.size() + n_threads - 1) / n_threads, 1);
        PDeltas tot(n_items, F, !low_mem);
        for (size_t c0 = 0; c0 < users.size(); c0 += chunk) {
            PDeltas d(n_items, F, !low_mem);
            std::vector<uint32_t> part(users.begin() + c0, users.begin() + std::min(users.size(), c0 + chunk));
            user_phase_p(tr, pr, part, d);
            for (size_t k = 0; k < d.dy.v.size(); ++k) tot.dy.v[k] += d.dy.v[k];
            for (size_t j = 0; j < n_items; ++j) {
                tot.dyb[j] += d.dyb[j];
                tot.nc[j] += d.nc[j];
            }
            if (!low_mem)
                for (size_t k = 0; k < d.dyd.v.size(); ++k) tot.dyd.v[k] += d.dyd.v[k];
        }
        apply_deltas_p(tr, pr, tot, nsvd_norm_exp);
    }

    // The epoch-start reset of the user factors (src/tsvdx4p.rs:401-404).
    void user_phase_prologue_p(uint64_t epoch) {
        if (epoch == cfg.reset_u_epoch) {
            ufeat.fill(T(0));
            ufeat2.fill(T(0));
        }
    }

    // The user phase for `users` in the given order, accumulating their NSVD1
    // deltas into d (src/tsvdx4p.rs:449-630, one chunk's loop).
    // With sv and se given (low_memory only), each user's delta row seq / norm
    // and sum_err / norm are written to sv[u * F ..] and se[u] instead of
    // being added into d, for a caller that sums them per item in user order.
    void user_phase_p(const DataView& tr, const DataView& pr, const std::vector<uint32_t>& users, PDeltas& d,
                      T* sv = nullptr, T* se = nullptr) {
        const Config c = cfg;
        const size_t F = c.n_feat, NF = c.n_freq_bins;
        const bool low_mem = c.low_memory, use_probe = c.full_su;
        (void)pr;
        std::vector<size_t> offs = calc_user_offsets(tr);
        const bool has_ud = !low_mem && c.lr_ud != 0.0f;
        Mat<T>& dy = d.dy;
        Mat<T>& dyd = d.dyd;
        std::vector<T>& dyb = d.dyb;
        std::vector<uint32_t>& nc = d.nc;
        {
            for (size_t ci = 0; ci < users.size(); ++ci) {
                const size_t u = users[ci];
                const size_t start = offs[u], end = offs[u + 1], cnt = end - start;
                if (cnt == 0) continue;
                std::vector<std::pair<size_t, size_t>> drs;
                if (!low_mem) drs = day_ranges(tr.dates, start, end);
                std::vector<T> su(F, T(0));
                T su_bias = T(0);
                for (size_t t = start; t < end; ++t) {
                    size_t j = tr.item_idxs[t];
                    for (size_t k = 0; k < F; ++k) su[k] += yfeat.at(j, k);
                    su_bias += ybias[j];
                }
                size_t total_cnt = cnt;
                if (use_probe) {
                    for (uint32_t j : probe_items_by_user[u]) {
                        for (size_t k = 0; k < F; ++k) su[k] += yfeat.at(j, k);
                        su_bias += ybias[j];
                    }
                    total_cnt = cnt + probe_items_by_user[u].size();
                }
                const T norm = sqrtT((T)(float)total_cnt);
                for (size_t k = 0; k < F; ++k) su[k] /= norm;
                su_bias /= norm;
                for (size_t k = 0; k < F; ++k) ycache.at(u, k) = su[k];
                ycache_bias[u] = su_bias;
                std::vector<T> seq(F, T(0)), seqd(F, T(0));
                T sum_err = T(0);
                std::vector<T> su_day(low_mem ? 0 : F, T(0));
                T norm_day = T(0);
                size_t dr_idx = 0, cur_f = 0;
                for (size_t t = start; t < end; ++t) {
                    const size_t i = tr.item_idxs[t];
                    const T r = (T)tr.residuals[t];
                    const int32_t day = tr.dates[t];
                    const int16_t day16 = tr.dates[t];
                    const size_t b = time_bin(day);
                    const T dv = dev(u, day);
                    size_t ds = 0, de = 0;
                    if (!low_mem) {
                        ds = drs[dr_idx].first;
                        de = drs[dr_idx].second;
                    }
                    if (!low_mem && t == ds) {
                        for (size_t k = 0; k < F; ++k) {
                            seqd[k] = T(0);
                            su_day[k] = T(0);
                        }
                        long idd = ud.index(u, day16);
                        cur_f = idd >= 0 ? freq_bin(ud.day_cnts[idd], NF) : 0;
                        for (size_t td = ds; td <= de; ++td)
                            for (size_t k = 0; k < F; ++k) su_day[k] += yfeat_day.at(tr.item_idxs[td], k);
                        float day_cnt = (float)(de - ds + 1);
                        if (use_probe && idd >= 0)
                            for (uint32_t j : probe_items_by_ud[idd]) {
                                for (size_t k = 0; k < F; ++k) su_day[k] += yfeat_day.at(j, k);
                                day_cnt += 1.0f;
                            }
                        norm_day = sqrtT((T)day_cnt);
                        for (size_t k = 0; k < F; ++k) su_day[k] /= norm_day;
                    }
                    const size_t f = cur_f;
                    const long idx = ud.index(u, day16);
                    const T ubias_u = ubias[u], but_ub = but_bin.at(u, b), alpha = alpha_u[u];
                    const T bu_day = idx >= 0 ? ubias_day[idx] : T(0);
                    const T cu_u = cu[u];
                    const T cu_t = cu_u + (idx >= 0 ? cut[idx] : T(0));
                    const T bu_t = ubias_u + but_ub + alpha * dv + bu_day + su_bias;
                    const T bi_t = ibias[i] + bit_bin.at(i, b) + ibias_freq.at(i, f);
                    T dot = T(0);
                    for (size_t k = 0; k < F; ++k) {
                        T qe = ifeat.at(i, k) + ifeat_freq.at(i * NF + f, k);
                        T pe = ufeat.at(u, k) + su[k] + dv * ufeat2.at(u, k);
                        if (!low_mem) {
                            if (has_ud && idx >= 0) pe += ufeat_day.at(idx, k);
                            pe += su_day[k];
                        }
                        dot += pe * qe;
                    }
                    const T score = gbias + bu_t + bi_t * cu_t + dot;
                    const T err = score - r;
                    ubias[u] -= (T)c.lr_ub * err;
                    but_bin.at(u, b) -= (T)c.lr_tu * err;
                    alpha_u[u] -= (T)c.lr_ta * err * dv;
                    if (idx >= 0) ubias_day[idx] -= (T)c.lr_ubd * err;
                    cu[u] -= (T)c.lr_cu * (err * bi_t + (T)c.reg_cu * (cu_u - T(1)));
                    sum_err += err;
                    for (size_t k = 0; k < F; ++k) {
                        T qe = ifeat.at(i, k) + ifeat_freq.at(i * NF + f, k);
                        T pu_k = ufeat.at(u, k), pu2_k = ufeat2.at(u, k);
                        seq[k] += err * qe;
                        if (!low_mem) seqd[k] += err * qe;
                        ufeat.at(u, k) -= (T)c.lr_u * (err * qe + (T)c.reg_u * pu_k);
                        ufeat2.at(u, k) -= (T)c.lr_u2 * (err * qe * dv + (T)c.reg_u2 * pu2_k);
                        if (has_ud && idx >= 0) {
                            T pud = ufeat_day.at(idx, k);
                            ufeat_day.at(idx, k) -= (T)c.lr_ud * (err * qe + (T)c.reg_ud * pud);
                        }
                    }
                    if (!low_mem && t == de) {
                        for (size_t td = ds; td <= de; ++td)
                            for (size_t k = 0; k < F; ++k) dyd.at(tr.item_idxs[td], k) += seqd[k] / norm_day;
                        ++dr_idx;
                    }
                }
                if (sv) {
                    for (size_t k = 0; k < F; ++k) sv[u * F + k] = seq[k] / norm;
                    se[u] = sum_err / norm;
                    continue;
                }
                for (size_t t = start; t < end; ++t) {
                    size_t j = tr.item_idxs[t];
                    for (size_t k = 0; k < F; ++k) dy.at(j, k) += seq[k] / norm;
                    dyb[j] += sum_err / norm;
                    nc[j] += 1;
                }
            }
        }
    }

    // fit_epoch_user_p with one chunk followed by fit_epoch_item_p, on
    // `workers` host threads, with the same arithmetic in the same order:
    // users' SGD in parallel slices of the epoch's order (item tables are
    // frozen in the user phase), each item's delta sum over the users in the
    // epoch's order (items split between the threads), the y update, the
    // cache rebuild per user (its train then probe rows in order) and the
    // item phase per item. low_memory only.
    void fit_epoch_p_workers(const DataView& tr, const DataView& pr, uint64_t epoch, float nsvd_norm_exp,
                             size_t workers) {
        const Config c = cfg;
        if (!c.low_memory) throw std::runtime_error("fit_epoch_p_workers: low_memory only");
        const size_t F = c.n_feat;
        workers = std::max<size_t>(workers, 1);
        auto par = [&](size_t n, auto&& body) {  // body(w, lo, hi) over n units in `workers` slices
            std::vector<std::thread> th;
            const size_t per = (n + workers - 1) / workers;
            for (size_t w = 0; w < workers; ++w) {
                const size_t lo = std::min(n, w * per), hi = std::min(n, lo + per);
                th.emplace_back([&, w, lo, hi] { body(w, lo, hi); });
            }
            for (auto& t : th) t.join();
        };
        user_phase_prologue_p(epoch);
        const std::vector<uint32_t> users = users_for_epoch(epoch);
        std::vector<T> sv(n_users * F, T(0)), se(n_users, T(0));
        par(users.size(), [&](size_t, size_t lo, size_t hi) {
            PDeltas scratch(0, F, false);
            std::vector<uint32_t> part(users.begin() + lo, users.begin() + hi);
            user_phase_p(tr, pr, part, scratch, sv.data(), se.data());
        });
        PDeltas tot(n_items, F, false);
        const std::vector<size_t> offs = calc_user_offsets(tr);
        par(n_items, [&](size_t, size_t j_lo, size_t j_hi) {
            for (uint32_t u : users)
                for (size_t t = offs[u]; t < offs[u + 1]; ++t) {
                    const size_t j = tr.item_idxs[t];
                    if (j < j_lo || j >= j_hi) continue;
                    for (size_t k = 0; k < F; ++k) tot.dy.at(j, k) += sv[u * F + k];
                    tot.dyb[j] += se[u];
                    tot.nc[j] += 1;
                }
        });
        apply_deltas_p_workers(tr, pr, tot, nsvd_norm_exp, par);
        if (by_item.starts.empty()) build_by_item(tr);
        std::vector<size_t> order(n_items);
        for (size_t i = 0; i < n_items; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
            return by_item.starts[x + 1] - by_item.starts[x] > by_item.starts[y + 1] - by_item.starts[y];
        });
        std::atomic<size_t> next{0};
        par(workers, [&](size_t, size_t, size_t) {
            for (size_t k; (k = next.fetch_add(1)) < n_items;) item_phase_p(tr, order[k], order[k] + 1);
        });
    }

    // apply_deltas_p with the cache rebuild split over users.
    template <class Par>
    void apply_deltas_p_workers(const DataView& tr, const DataView& pr, const PDeltas& tot, float nsvd_norm_exp,
                                Par&& par) {
        const Config c = cfg;
        const size_t F = c.n_feat;
        const float ex = nsvd_norm_exp;
        for (size_t j = 0; j < n_items; ++j) {
            if (tot.nc[j] == 0) continue;
            T scale = ex == 0.0f ? T(1) : powT((T)(float)tot.nc[j], (T)ex);
            for (size_t k = 0; k < F; ++k) {
                T yj = yfeat.at(j, k);
                yfeat.at(j, k) -= (T)c.lr_y * (tot.dy.at(j, k) / scale + (T)c.reg_y * yj);
            }
            ybias[j] -= (T)c.lr_yb * (tot.dyb[j] / scale);
        }
        // each user's train rows, then its probe rows, in row order (the
        // probe set need not be user-sorted)
        std::vector<size_t> off(n_users + 1, 0);
        for (size_t t = 0; t < tr.n_ratings; ++t) ++off[tr.user_idxs[t] + 1];
        for (size_t t = 0; t < pr.n_ratings; ++t) ++off[pr.user_idxs[t] + 1];
        for (size_t u = 0; u < n_users; ++u) off[u + 1] += off[u];
        std::vector<uint32_t> items(off[n_users]);
        {
            std::vector<size_t> at(off.begin(), off.end() - 1);
            for (size_t t = 0; t < tr.n_ratings; ++t) items[at[tr.user_idxs[t]]++] = (uint32_t)tr.item_idxs[t];
            for (size_t t = 0; t < pr.n_ratings; ++t) items[at[pr.user_idxs[t]]++] = (uint32_t)pr.item_idxs[t];
        }
        par(n_users, [&](size_t, size_t u_lo, size_t u_hi) {
            for (size_t u = u_lo; u < u_hi; ++u) {
                T* su = ycache.row(u);
                T sb = T(0);
                for (size_t k = 0; k < F; ++k) su[k] = T(0);
                for (size_t e = off[u]; e < off[u + 1]; ++e) {
                    const T* y = yfeat.row(items[e]);
                    for (size_t k = 0; k < F; ++k) su[k] += y[k];
                    sb += ybias[items[e]];
                }
                const int32_t cnt = tr.user_cnts[u] + pr.user_cnts[u];
                if (cnt > 0) {
                    const T nrm = sqrtT((T)(float)cnt);
                    for (size_t k = 0; k < F; ++k) su[k] /= nrm;
                    sb /= nrm;
                }
                ycache_bias[u] = sb;
            }
        });
    }

    // apply_nsvd_deltas (src/tsvdx4p.rs:341-385) of the summed deltas, then
    // the cache rebuild (:636-638).
    void apply_deltas_p(const DataView& tr, const DataView& pr, const PDeltas& tot, float nsvd_norm_exp) {
        const Config c = cfg;
        const size_t F = c.n_feat;
        const bool low_mem = c.low_memory;
        const Mat<T>& tot_dy = tot.dy;
        const Mat<T>& tot_dyd = tot.dyd;
        const std::vector<T>& tot_dyb = tot.dyb;
        const std::vector<uint32_t>& tot_nc = tot.nc;
        const float ex = nsvd_norm_exp;
        for (size_t j = 0; j < n_items; ++j) {
            if (tot_nc[j] == 0) continue;
            T scale = ex == 0.0f ? T(1) : powT((T)(float)tot_nc[j], (T)ex);
            for (size_t k = 0; k < F; ++k) {
                T yj = yfeat.at(j, k);
                yfeat.at(j, k) -= (T)c.lr_y * (tot_dy.at(j, k) / scale + (T)c.reg_y * yj);
            }
            ybias[j] -= (T)c.lr_yb * (tot_dyb[j] / scale);
        }
        if (!low_mem)
            for (size_t j = 0; j < n_items; ++j) {
                if (tot_nc[j] == 0) continue;
                T scale = ex == 0.0f ? T(1) : powT((T)(float)tot_nc[j], (T)ex);
                for (size_t k = 0; k < F; ++k) {
                    T yj = yfeat_day.at(j, k);
                    yfeat_day.at(j, k) -= (T)c.lr_yd * (tot_dyd.at(j, k) / scale + (T)c.reg_yd * yj);
                }
            }
        rebuild_ycache(tr, pr);
        if (!low_mem) rebuild_ycache_day(tr, pr);
    }

    // src/tsvdx4p.rs:644-762
    void fit_epoch_item_p(const DataView& tr) { item_phase_p(tr, 0, n_items); }

    // The item phase for items i_lo..i_hi-1.
    void item_phase_p(const DataView& tr, size_t i_lo, size_t i_hi) {
        const Config c = cfg;
        const size_t F = c.n_feat, NF = c.n_freq_bins;
        const bool low_mem = c.low_memory;
        if (by_item.starts.empty()) build_by_item(tr);
        std::vector<T> pe(F);
        for (size_t i = i_lo; i < i_hi; ++i) {
            for (size_t e = by_item.starts[i]; e < by_item.starts[i + 1]; ++e) {
                const size_t u = by_item.user[e], t = by_item.rating[e];
                const T r = (T)tr.residuals[t];
                const int32_t day = tr.dates[t];
                const size_t b = time_bin(day);
                const T dv = dev(u, day);
                const long idx = ud.index(u, tr.dates[t]);
                const size_t f = idx >= 0 ? freq_bin(ud.day_cnts[idx], NF) : 0;
                const T bu_day = idx >= 0 ? ubias_day[idx] : T(0);
                const T bu_t = ubias[u] + but_bin.at(u, b) + alpha_u[u] * dv + bu_day + ycache_bias[u];
                const T bi_t = ibias[i] + bit_bin.at(i, b) + ibias_freq.at(i, f);
                const T cu_t = cu[u] + (idx >= 0 ? cut[idx] : T(0));
                T dot = T(0);
                for (size_t k = 0; k < F; ++k) {
                    T qe = ifeat.at(i, k) + ifeat_freq.at(i * NF + f, k);
                    T p = ufeat.at(u, k) + ycache.at(u, k) + dv * ufeat2.at(u, k);
                    if (!low_mem && idx >= 0) {
                        p += ufeat_day.at(idx, k);
                        p += ycache_day.at(idx, k);
                    }
                    pe[k] = p;
                    dot += p * qe;
                }
                const T score = gbias + bu_t + bi_t * cu_t + dot;
                const T err = score - r;
                ibias[i] -= (T)c.lr_ib * (err * cu_t);
                bit_bin.at(i, b) -= (T)c.lr_ti * (err * cu_t);
                ibias_freq.at(i, f) -= (T)c.lr_ibf * (err * cu_t);
                for (size_t k = 0; k < F; ++k) {
                    T qi_k = ifeat.at(i, k), qf_k = ifeat_freq.at(i * NF + f, k);
                    ifeat.at(i, k) -= (T)c.lr_i * (err * pe[k] + (T)c.reg_i * qi_k);
                    ifeat_freq.at(i * NF + f, k) -= (T)c.lr_iqf * (err * pe[k] + (T)c.reg_iqf * qf_k);
                }
            }
        }
    }
};

// calc_rmse (src/lib.rs:659-672): FP64 SSE over is_test == 0 rows.
template <class M>
double calc_rmse(const M& m, const DataView& ds) {
    double cnt = 0.0, sse = 0.0;
    for (size_t t = 0; t < ds.n_ratings; ++t) {
        if (ds.is_test[t] != 0) continue;
        using T = decltype(m.gbias);
        T d = m.predict(ds.user_idxs[t], ds.item_idxs[t], ds.dates[t]) - (T)ds.residuals[t];
        double err = (double)d;
        cnt += 1.0;
        sse += err * err;
    }
    return std::sqrt(sse / cnt);
}

}  // namespace oracle
