// TEST INFRASTRUCTURE ONLY -- C entry points of the CPU oracle, loaded with
// ctypes by the tests, the smoke check and bench.py's CPU-baseline leg. It
// shares the struct layouts of include/tsvdx4_cuda.h so one Python config
// object feeds both the oracle and the CUDA library.
#include <chrono>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../include/tsvdx4_cuda.h"
#include "tx_oracle.hpp"

using namespace oracle;

namespace {

thread_local std::string g_err;

Config to_cfg(const tsvd_config& c) {
    Config o{};
    o.n_feat = c.n_feat;
    o.n_epochs = c.n_epochs;
    o.seed = c.seed;
    o.shuffle_users = c.shuffle_users != 0;
    o.n_time_bins = c.n_time_bins;
    o.beta = c.beta;
    o.n_freq_bins = c.n_freq_bins;
    o.lr_u = c.lr_u; o.lr_ud = c.lr_ud; o.lr_u2 = c.lr_u2; o.lr_ub = c.lr_ub; o.lr_ubd = c.lr_ubd;
    o.lr_i = c.lr_i; o.lr_ib = c.lr_ib; o.lr_y = c.lr_y; o.lr_yb = c.lr_yb; o.lr_yd = c.lr_yd;
    o.lr_tu = c.lr_tu; o.lr_ti = c.lr_ti; o.lr_ta = c.lr_ta; o.lr_ibf = c.lr_ibf; o.lr_iqf = c.lr_iqf;
    o.lr_cu = c.lr_cu;
    o.reg_iqf = c.reg_iqf; o.reg_cu = c.reg_cu; o.reg_u = c.reg_u; o.reg_u2 = c.reg_u2; o.reg_ud = c.reg_ud;
    o.reg_i = c.reg_i; o.reg_y = c.reg_y; o.reg_yd = c.reg_yd;
    o.sigma_iqf = c.sigma_iqf; o.sigma_u = c.sigma_u; o.sigma_i = c.sigma_i; o.sigma_y = c.sigma_y;
    o.sigma_yd = c.sigma_yd;
    o.reset_u_epoch = c.reset_u_epoch;
    o.max_neighbors = c.max_neighbors;
    o.lr_w = c.lr_w; o.lr_c = c.lr_c; o.reg_w = c.reg_w; o.reg_c = c.reg_c;
    o.lr_w_day = c.lr_w_day; o.lr_c_day = c.lr_c_day; o.reg_w_day = c.reg_w_day; o.reg_c_day = c.reg_c_day;
    o.w_bias = c.w_bias; o.w_factor = c.w_factor; o.w_nbr = c.w_nbr;
    o.sum_err_bug = c.sum_err_bug != 0;
    o.lambda1 = c.lambda1; o.lambda2 = c.lambda2;
    o.has_ordinal = c.has_ordinal_head != 0;
    std::memcpy(o.ordinal.th_init, c.ordinal_head.th_init, sizeof(o.ordinal.th_init));
    o.ordinal.th_gap = c.ordinal_head.th_gap;
    o.ordinal.lr_t = c.ordinal_head.lr_t;
    o.ordinal.reg_t = c.ordinal_head.reg_t;
    o.save_ifeat = c.save_ifeat != 0;
    o.low_memory = c.low_memory != 0;
    o.full_su = c.full_su != 0;
    return o;
}

DataView to_view(const tsvd_dataset_view& d) {
    return DataView{d.user_idxs, d.user_cnts, d.item_idxs, d.raw_ratings, d.residuals,
                    d.dates,     d.is_test,   (size_t)d.n_users, (size_t)d.n_items, (size_t)d.n_ratings};
}

// Owns private copies of both datasets so the Python side may drop its arrays.
struct OwnedData {
    std::vector<int32_t> u, uc, i;
    std::vector<int8_t> raw, tst;
    std::vector<float> res;
    std::vector<int16_t> d;
    DataView v{};
    void take(const tsvd_dataset_view& s) {
        size_t n = s.n_ratings;
        u.assign(s.user_idxs, s.user_idxs + n);
        uc.assign(s.user_cnts, s.user_cnts + s.n_users);
        i.assign(s.item_idxs, s.item_idxs + n);
        d.assign(s.dates, s.dates + n);
        if (s.raw_ratings) raw.assign(s.raw_ratings, s.raw_ratings + n);
        if (s.residuals) res.assign(s.residuals, s.residuals + n);
        if (s.is_test) tst.assign(s.is_test, s.is_test + n); else tst.assign(n, 0);
        v = DataView{u.data(), uc.data(), i.data(), raw.empty() ? nullptr : raw.data(),
                     res.empty() ? nullptr : res.data(), d.data(), tst.data(), (size_t)s.n_users,
                     (size_t)s.n_items, n};
    }
};

struct Handle {
    OwnedData tr, pr;
    bool fp64 = false;
    std::unique_ptr<TxModel<float>> m32;
    std::unique_ptr<TxModel<double>> m64;
};

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

template <class M>
bool param_ptr(M& m, const std::string& n, void*& p, size_t& count, bool& is_scalar) {
    is_scalar = false;
    auto vec = [&](auto& v) { p = v.data(); count = v.size(); return true; };
    auto mat = [&](auto& mm) { p = mm.v.data(); count = mm.v.size(); return true; };
    if (n == "gbias") { p = &m.gbias; count = 1; is_scalar = true; return true; }
    if (n == "ubias") return vec(m.ubias);
    if (n == "ibias") return vec(m.ibias);
    if (n == "ufeat") return mat(m.ufeat);
    if (n == "ufeat2") return mat(m.ufeat2);
    if (n == "ifeat") return mat(m.ifeat);
    if (n == "yfeat") return mat(m.yfeat);
    if (n == "ycache") return mat(m.ycache);
    if (n == "yfeat_day") return mat(m.yfeat_day);
    if (n == "tu_mean") return vec(m.tu_mean);
    if (n == "alpha_u") return vec(m.alpha_u);
    if (n == "but_bin") return mat(m.but_bin);
    if (n == "bit_bin") return mat(m.bit_bin);
    if (n == "ybias") return vec(m.ybias);
    if (n == "ycache_bias") return vec(m.ycache_bias);
    if (n == "ubias_day") return vec(m.ubias_day);
    if (n == "ufeat_day") return mat(m.ufeat_day);
    if (n == "ycache_day") return mat(m.ycache_day);
    if (n == "ibias_freq") return mat(m.ibias_freq);
    if (n == "ifeat_freq") return mat(m.ifeat_freq);
    if (n == "cu") return vec(m.cu);
    if (n == "cut") return vec(m.cut);
    return false;
}

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const tsvd_config* cfg, const tsvd_dataset_view* tr, const tsvd_dataset_view* pr, int fp64) {
    Handle* h = new Handle();
    int rc = guard([&] {
        h->tr.take(*tr);
        h->pr.take(*pr);
        h->fp64 = fp64 != 0;
        Config c = to_cfg(*cfg);
        if (h->fp64) h->m64.reset(new TxModel<double>(h->tr.v, h->pr.v, c));
        else h->m32.reset(new TxModel<float>(h->tr.v, h->pr.v, c));
    });
    if (rc) {
        delete h;
        return nullptr;
    }
    return h;
}

void orc_destroy(void* p) { delete (Handle*)p; }

// schedule: 0 = TxModel::fit_epoch (sequential reference);
//           1 = Tsvdx4pModel parallel epoch (user phase then item phase).
int orc_fit_epoch(void* p, uint64_t epoch, int schedule, float nsvd_norm_exp, uint64_t n_threads) {
    Handle* h = (Handle*)p;
    return guard([&] {
        auto run = [&](auto& m) {
            if (schedule == 0) {
                m.fit_epoch(h->tr.v, h->pr.v, epoch);
            } else if (schedule == 1) {
                m.fit_epoch_user_p(h->tr.v, h->pr.v, epoch, nsvd_norm_exp, n_threads);
                m.fit_epoch_item_p(h->tr.v);
            } else {
                throw std::runtime_error("unknown schedule");
            }
        };
        if (h->fp64) run(*h->m64); else run(*h->m32);
    });
}

// Schedule 1 with one chunk (n_threads = 1), computed on `workers` host
// threads; the same arithmetic in the same order (low_memory only).
int orc_fit_epoch_p_workers(void* p, uint64_t epoch, float nsvd_norm_exp, uint64_t workers) {
    Handle* h = (Handle*)p;
    return guard([&] {
        if (h->fp64) h->m64->fit_epoch_p_workers(h->tr.v, h->pr.v, epoch, nsvd_norm_exp, workers);
        else h->m32->fit_epoch_p_workers(h->tr.v, h->pr.v, epoch, nsvd_norm_exp, workers);
    });
}

// The parallel schedule in the steps a sharded run takes (src/tsvdx4p.rs:
// fit_epoch_user :390-639 restricted to the users u_lo..u_hi-1, in the epoch's
// order; apply_nsvd_deltas :341-385 of deltas summed elsewhere; fit_epoch_item
// :644-762 restricted to items i_lo..i_hi-1). Deltas cross the boundary as
// FP64 arrays: dy [I*F], dyb [I], dyd [I*F] (low_memory = false, else NULL),
// nc [I].
int orc_user_block_p(void* p, uint64_t epoch, uint64_t u_lo, uint64_t u_hi, double* dy, double* dyb, double* dyd,
                     double* nc) {
    Handle* h = (Handle*)p;
    return guard([&] {
        auto run = [&](auto& m) {
            using M = std::remove_reference_t<decltype(m)>;
            m.user_phase_prologue_p(epoch);
            std::vector<uint32_t> users;
            for (uint32_t u : m.users_for_epoch(epoch))
                if (u >= u_lo && u < u_hi) users.push_back(u);
            typename M::PDeltas d(m.n_items, m.cfg.n_feat, !m.cfg.low_memory);
            m.user_phase_p(h->tr.v, h->pr.v, users, d);
            for (size_t k = 0; k < d.dy.v.size(); ++k) dy[k] = (double)d.dy.v[k];
            for (size_t j = 0; j < m.n_items; ++j) {
                dyb[j] = (double)d.dyb[j];
                nc[j] = (double)d.nc[j];
            }
            if (!m.cfg.low_memory)
                for (size_t k = 0; k < d.dyd.v.size(); ++k) dyd[k] = (double)d.dyd.v[k];
        };
        if (h->fp64) run(*h->m64); else run(*h->m32);
    });
}

int orc_apply_deltas_p(void* p, const double* dy, const double* dyb, const double* dyd, const double* nc,
                       float nsvd_norm_exp) {
    Handle* h = (Handle*)p;
    return guard([&] {
        auto run = [&](auto& m) {
            using M = std::remove_reference_t<decltype(m)>;
            using T = std::remove_reference_t<decltype(m.ubias[0])>;
            typename M::PDeltas d(m.n_items, m.cfg.n_feat, !m.cfg.low_memory);
            for (size_t k = 0; k < d.dy.v.size(); ++k) d.dy.v[k] = (T)dy[k];
            for (size_t j = 0; j < m.n_items; ++j) {
                d.dyb[j] = (T)dyb[j];
                d.nc[j] = (uint32_t)nc[j];
            }
            if (!m.cfg.low_memory)
                for (size_t k = 0; k < d.dyd.v.size(); ++k) d.dyd.v[k] = (T)dyd[k];
            m.apply_deltas_p(h->tr.v, h->pr.v, d, nsvd_norm_exp);
        };
        if (h->fp64) run(*h->m64); else run(*h->m32);
    });
}

int orc_item_block_p(void* p, uint64_t i_lo, uint64_t i_hi) {
    Handle* h = (Handle*)p;
    return guard([&] {
        if (h->fp64) h->m64->item_phase_p(h->tr.v, i_lo, i_hi);
        else h->m32->item_phase_p(h->tr.v, i_lo, i_hi);
    });
}

int orc_predict(void* p, const int32_t* u, const int32_t* i, const int16_t* day, uint64_t n, double* out) {
    Handle* h = (Handle*)p;
    return guard([&] {
        for (uint64_t k = 0; k < n; ++k)
            out[k] = h->fp64 ? h->m64->predict(u[k], i[k], day[k]) : (double)h->m32->predict(u[k], i[k], day[k]);
    });
}

int orc_predict_subscores(void* p, const int32_t* u, const int32_t* i, const int16_t* day, uint64_t n,
                          double* out) {
    Handle* h = (Handle*)p;
    return guard([&] {
        for (uint64_t k = 0; k < n; ++k) {
            if (h->fp64) {
                double s[3];
                h->m64->predict_subscores(u[k], i[k], day[k], s);
                for (int c = 0; c < 3; ++c) out[3 * k + c] = s[c];
            } else {
                float s[3];
                h->m32->predict_subscores(u[k], i[k], day[k], s);
                for (int c = 0; c < 3; ++c) out[3 * k + c] = s[c];
            }
        }
    });
}

int orc_calc_rmse(void* p, const tsvd_dataset_view* ds, double* out) {
    Handle* h = (Handle*)p;
    return guard([&] {
        DataView v = to_view(*ds);
        *out = h->fp64 ? calc_rmse(*h->m64, v) : calc_rmse(*h->m32, v);
    });
}

int orc_rebuild_ycache(void* p) {
    Handle* h = (Handle*)p;
    return guard([&] {
        if (h->fp64) {
            h->m64->rebuild_ycache(h->tr.v, h->pr.v);
            if (!h->m64->cfg.low_memory) h->m64->rebuild_ycache_day(h->tr.v, h->pr.v);
        } else {
            h->m32->rebuild_ycache(h->tr.v, h->pr.v);
            if (!h->m32->cfg.low_memory) h->m32->rebuild_ycache_day(h->tr.v, h->pr.v);
        }
    });
}

// Parameters travel as f64 arrays (lossless for the f32 model).
int orc_param_count(void* p, const char* name, uint64_t* out) {
    Handle* h = (Handle*)p;
    return guard([&] {
        void* ptr; size_t cnt; bool sc;
        bool ok = h->fp64 ? param_ptr(*h->m64, name, ptr, cnt, sc) : param_ptr(*h->m32, name, ptr, cnt, sc);
        if (std::string(name) == "thresholds") { *out = 4; return; }
        if (!ok) throw std::runtime_error(std::string("unknown parameter ") + name);
        *out = cnt;
    });
}

int orc_get_param(void* p, const char* name, double* dst, uint64_t count) {
    Handle* h = (Handle*)p;
    return guard([&] {
        if (std::string(name) == "thresholds") {
            const float* th = h->fp64 ? h->m64->ordinal.th : h->m32->ordinal.th;
            for (int k = 0; k < 4 && k < (int)count; ++k) dst[k] = th[k];
            return;
        }
        void* ptr; size_t cnt; bool sc;
        bool ok = h->fp64 ? param_ptr(*h->m64, name, ptr, cnt, sc) : param_ptr(*h->m32, name, ptr, cnt, sc);
        if (!ok) throw std::runtime_error(std::string("unknown parameter ") + name);
        if (cnt != count) throw std::runtime_error("count mismatch for " + std::string(name));
        for (size_t k = 0; k < cnt; ++k) dst[k] = h->fp64 ? ((double*)ptr)[k] : (double)((float*)ptr)[k];
    });
}

int orc_set_param(void* p, const char* name, const double* src, uint64_t count) {
    Handle* h = (Handle*)p;
    return guard([&] {
        void* ptr; size_t cnt; bool sc;
        bool ok = h->fp64 ? param_ptr(*h->m64, name, ptr, cnt, sc) : param_ptr(*h->m32, name, ptr, cnt, sc);
        if (!ok) throw std::runtime_error(std::string("unknown parameter ") + name);
        if (cnt != count) throw std::runtime_error("count mismatch for " + std::string(name));
        for (size_t k = 0; k < cnt; ++k) {
            if (h->fp64) ((double*)ptr)[k] = src[k];
            else ((float*)ptr)[k] = (float)src[k];
        }
    });
}

int orc_set_user_order(void* p, uint64_t epoch, const uint32_t* perm, uint64_t n) {
    Handle* h = (Handle*)p;
    return guard([&] {
        auto set = [&](auto& m) {
            if (n != m.n_users) throw std::runtime_error("permutation length != n_users");
            if (m.injected_order.size() <= epoch) m.injected_order.resize(epoch + 1);
            m.injected_order[epoch].assign(perm, perm + n);
        };
        if (h->fp64) set(*h->m64); else set(*h->m32);
    });
}

// get_users (src/lib.rs:486-494) through the restated rand 0.9 shuffle.
int orc_get_users(uint64_t n, int shuffle, uint64_t seed, uint64_t epoch, uint32_t* out) {
    return guard([&] {
        std::vector<uint32_t> u = get_users(n, shuffle != 0, seed, epoch);
        std::memcpy(out, u.data(), n * sizeof(uint32_t));
    });
}

// First `n` f32 draws of rand_array2 from StdRng(seed) with the given sigma.
int orc_normal_stream(uint64_t seed, float sigma, uint64_t n, float* out) {
    return guard([&] {
        StdRng rng = StdRng::seed_from_u64(seed);
        for (uint64_t k = 0; k < n; ++k) out[k] = normal_f32(rng, sigma);
    });
}

// Raw u32 words of StdRng(seed).
int orc_u32_stream(uint64_t seed, uint64_t n, uint32_t* out) {
    return guard([&] {
        StdRng rng = StdRng::seed_from_u64(seed);
        for (uint64_t k = 0; k < n; ++k) out[k] = rng.next_u32();
    });
}

// One ChaCha block with the given rounds over a caller-supplied state.
void orc_chacha_block(const uint32_t* in, uint32_t* out, int rounds) { chacha_block(in, out, rounds); }

// Seconds of wall time for `epochs` sequential epochs (CPU baseline).
int orc_time_epochs(void* p, uint64_t first_epoch, uint64_t epochs, int schedule, double* seconds) {
    Handle* h = (Handle*)p;
    auto t0 = std::chrono::steady_clock::now();
    for (uint64_t e = 0; e < epochs; ++e) {
        int rc = orc_fit_epoch(p, first_epoch + e, schedule, 1.0f, 1);
        if (rc) return rc;
    }
    (void)h;
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

}  // extern "C"
