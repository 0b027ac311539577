// extern "C" entry points declared in include/tsvdx4_cuda.h.
#include <cstring>
#include <string>

#include "rand_stream.hpp"
#include "tsvd_model.hpp"

using tsvd::Error;

namespace tsvd {
std::string& global_err() {
    thread_local std::string e;
    return e;
}
}  // namespace tsvd

namespace {

using tsvd::guarded;
using tsvd::use_device;

struct ParamRef {
    float* dev;
    size_t rows, cols, stride;  // in floats
};

bool find_param(const tsvd_model* m, const std::string& n, ParamRef& r) {
    const tsvd::DeviceState& s = m->d;
    const size_t U = s.n_users, I = s.n_items, F = s.F, Fs = s.Fs, T = s.T, NF = s.NF, UD = s.n_ud;
    auto set = [&](float* p, size_t rows, size_t cols, size_t stride) {
        r = ParamRef{p, rows, cols, stride};
        return true;
    };
    if (n == "ubias") return set(s.ubias, 1, U, U);
    if (n == "ibias") return set(s.ibias, 1, I, I);
    if (n == "ufeat") return set(s.ufeat, U, F, Fs);
    if (n == "ufeat2") return set(s.ufeat2, U, F, Fs);
    if (n == "ifeat") return set(s.ifeat, I, F, Fs);
    if (n == "yfeat") return set(s.yfeat, I, F, Fs);
    if (n == "ycache") return set(s.ycache, U, F, Fs);
    if (n == "tu_mean") return set(const_cast<float*>(s.tu_mean), 1, U, U);
    if (n == "alpha_u") return set(s.alpha_u, 1, U, U);
    if (n == "but_bin") return set(s.but_bin, U, T, T);
    if (n == "bit_bin") return set(s.bit_bin, I, T, T);
    if (n == "ybias") return set(s.ybias, 1, I, I);
    if (n == "ycache_bias") return set(s.ycache_bias, 1, U, U);
    if (n == "ubias_day") return set(s.ubias_day, 1, UD, UD);
    if (n == "yfeat_day" && s.yfeat_day) return set(s.yfeat_day, I, F, Fs);
    if (n == "ufeat_day" && s.ufeat_day) return set(s.ufeat_day, UD, F, Fs);
    if (n == "ycache_day" && s.ycache_day) return set(s.ycache_day, UD, F, Fs);
    if (n == "ibias_freq") return set(s.ibias_freq, I, NF, NF);
    if (n == "ifeat_freq") return set(s.ifeat_freq, I * NF, F, Fs);
    if (n == "cu") return set(s.cu, 1, U, U);
    if (n == "cut") return set(s.cut, 1, UD, UD);
    return false;
}

const char* kSubscoreNames[3] = {"bias", "mf", "nsvd1"};

// Device copies of a call's host row columns in the model's staging buffer:
// reserve() sizes it for the call, put() copies one column (256-byte aligned
// slots), out() hands out an uninitialised slot.
struct RowStage {
    char* base = nullptr;
    size_t off = 0;
    static size_t slot(size_t bytes) { return (bytes + 255) / 256 * 256; }
    RowStage(const tsvd_model* m, size_t bytes) {
        if (m->m_rows.bytes < bytes) m->m_rows.alloc(bytes);
        base = m->m_rows.as<char>();
    }
    template <class T>
    const T* put(const T* h, uint64_t n, cudaStream_t st) {
        if (!h) return nullptr;
        T* d = reinterpret_cast<T*>(base + off);
        TSVD_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
        off += slot(n * sizeof(T));
        return d;
    }
    template <class T>
    T* out(uint64_t n) {
        T* d = reinterpret_cast<T*>(base + off);
        off += slot(n * sizeof(T));
        return d;
    }
};

}  // namespace

namespace tsvd {

void prof_begin(tsvd_model* m, const char* name, cudaEvent_t* ev) {
    if (!m->profiling) return;
    TSVD_CUDA(cudaEventCreate(&ev[0]));
    TSVD_CUDA(cudaEventCreate(&ev[1]));
    TSVD_CUDA(cudaEventRecord(ev[0], m->stream));
}

void prof_end(tsvd_model* m, const char* name, cudaEvent_t* ev) {
    if (!m->profiling || !ev[0]) return;
    cudaEventRecord(ev[1], m->stream);
    m->pending.push_back({name, {ev[0], ev[1]}});
}

static void drain_stats(tsvd_model* m) {
    for (auto& pe : m->pending) {
        cudaEventSynchronize(pe.second.second);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
        KernelStat& ks = m->stats[pe.first];
        ks.launches++;
        ks.total_ms += ms;
        cudaEventDestroy(pe.second.first);
        cudaEventDestroy(pe.second.second);
    }
    m->pending.clear();
}

}  // namespace tsvd

extern "C" {

int tsvd_abi_version(void) { return TSVD_ABI_VERSION; }

const char* tsvd_last_global_error(void) { return tsvd::global_err().c_str(); }

const char* tsvd_last_error(const tsvd_model* m) { return m ? m->err.c_str() : tsvd::global_err().c_str(); }

int tsvd_create(const tsvd_config* cfg, const tsvd_gpu_options* opts, const tsvd_dataset_view* tr,
                const tsvd_dataset_view* pr, tsvd_model** out) {
    if (!out) return TSVD_ERR_INVALID;
    *out = nullptr;
    tsvd_model* m = new tsvd_model();
    int rc = guarded(m, [&] {
        if (!cfg || !tr || !pr) throw Error(TSVD_ERR_INVALID, "null config or dataset view");
        m->cfg = *cfg;
        if (opts) m->opts = *opts;
        else {
            std::memset(&m->opts, 0, sizeof(m->opts));
            m->opts.nsvd_norm_exp = 1.0f;
        }
        if (m->opts.schedule != TSVD_SCHED_HOGWILD && m->opts.schedule != TSVD_SCHED_STRATIFIED &&
            m->opts.schedule != TSVD_SCHED_SEQUENTIAL)
            throw Error(TSVD_ERR_INVALID, "unknown schedule");
        if (m->opts.precision < TSVD_PREC_FP32 || m->opts.precision > TSVD_PREC_BF16_READ_ALL)
            throw Error(TSVD_ERR_INVALID, "unknown precision");
        if (m->opts.precision != TSVD_PREC_FP32 && m->opts.schedule != TSVD_SCHED_STRATIFIED)
            throw Error(TSVD_ERR_UNSUPPORTED,
                        "BF16 read copies need the stratified schedule (Hogwild writes the tables it reads)");
        if (m->opts.heavy_item_ratings < 0) throw Error(TSVD_ERR_INVALID, "heavy_item_ratings must be >= 0");
        int n_dev = 0;
        if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
            throw Error(TSVD_ERR_NO_DEVICE, "no CUDA device is visible");
        if (m->opts.device < 0 || m->opts.device >= n_dev) throw Error(TSVD_ERR_NO_DEVICE, "device ordinal out of range");
        m->device = m->opts.device;
        TSVD_CUDA(cudaSetDevice(m->device));
        cudaDeviceProp prop;
        TSVD_CUDA(cudaGetDeviceProperties(&prop, m->device));
        if (prop.major < 10) throw Error(TSVD_ERR_NO_DEVICE, "an sm_100 (Blackwell) device is required");
        TSVD_CUDA(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking));
        m->stream = m->own_stream;
        tsvd::setup_model(m, *tr, *pr);
    });
    if (rc != TSVD_OK) {
        tsvd::global_err() = m->err;
        tsvd_destroy(m);
        return rc;
    }
    *out = m;
    return TSVD_OK;
}

void tsvd_destroy(tsvd_model* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (auto& pe : m->pending) {
        cudaEventDestroy(pe.second.first);
        cudaEventDestroy(pe.second.second);
    }
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
    delete m;
}

int tsvd_n_epochs(const tsvd_model* m, uint64_t* out) {
    if (!m || !out) return TSVD_ERR_INVALID;
    *out = m->cfg.n_epochs;
    return TSVD_OK;
}

int tsvd_fit_epoch(tsvd_model* m, uint64_t epoch) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (epoch == 0) throw Error(TSVD_ERR_INVALID, "epochs are 1-based");
        use_device(m);
        tsvd::run_epoch(m, epoch);
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int tsvd_predict_batch_device(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day, uint64_t n,
                              float* out) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        use_device(m);
        tsvd::predict_device(m, u, i, day, nullptr, n, out, 0);
    });
}

static void check_rows(const tsvd_model* m, const int32_t* u, const int32_t* i, uint64_t n) {
    // in parallel; a failure reruns the check in row order for the first bad row
    const uint32_t U = m->d.n_users, I = m->d.n_items;
    bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok) if (n > 65536)
    for (int64_t k = 0; k < (int64_t)n; ++k)
        ok = ok && u[k] >= 0 && (uint32_t)u[k] < U && i[k] >= 0 && (uint32_t)i[k] < I;
    if (ok) return;
    for (uint64_t k = 0; k < n; ++k)
        if (u[k] < 0 || (uint32_t)u[k] >= m->d.n_users || i[k] < 0 || (uint32_t)i[k] >= m->d.n_items)
            throw Error(TSVD_ERR_INVALID, "row " + std::to_string(k) + ": user or item index out of range");
}

static int predict_host(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day,
                        const float* offset, uint64_t n, float* out, int subscores) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (n == 0) return;
        if (!u || !i || !day || !out) throw Error(TSVD_ERR_INVALID, "null row array");
        check_rows(m, u, i, n);
        use_device(m);
        cudaStream_t st = m->stream;
        const uint64_t cols = subscores ? 3 : 1;
        RowStage rs(m, 2 * RowStage::slot(n * 4) + RowStage::slot(n * 2) + RowStage::slot(n * 4) +
                           RowStage::slot(n * cols * 4));
        const int32_t* du = rs.put(u, n, st);
        const int32_t* di = rs.put(i, n, st);
        const int16_t* dd = rs.put(day, n, st);
        const float* doff = rs.put(offset, n, st);
        float* dout = rs.out<float>(n * cols);
        tsvd::predict_device(m, du, di, dd, doff, n, dout, subscores);
        TSVD_CUDA(cudaMemcpyAsync(out, dout, n * cols * sizeof(float), cudaMemcpyDeviceToHost, st));
        TSVD_CUDA(cudaStreamSynchronize(st));
    });
}

int tsvd_predict_batch(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day, uint64_t n,
                       float* out) {
    return predict_host(m, u, i, day, nullptr, n, out, 0);
}

int tsvd_n_subscores(const tsvd_model* m, uint64_t* out) {
    if (!m || !out) return TSVD_ERR_INVALID;
    *out = 3;
    return TSVD_OK;
}

const char* tsvd_subscore_name(const tsvd_model* m, uint64_t k) { return (m && k < 3) ? kSubscoreNames[k] : nullptr; }

int tsvd_predict_subscores_batch(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day,
                                 uint64_t n, float* out) {
    return predict_host(m, u, i, day, nullptr, n, out, 1);
}

int tsvd_gen_preds(const tsvd_model* m, const tsvd_dataset_view* ds, float* out) {
    if (!m || !ds) return TSVD_ERR_INVALID;
    if (!ds->raw_ratings || !ds->residuals) {
        m->err = "gen_preds needs a full view (raw_ratings and residuals)";
        return TSVD_ERR_INVALID;
    }
    std::vector<float> off(ds->n_ratings);
    for (uint64_t k = 0; k < ds->n_ratings; ++k) off[k] = (float)ds->raw_ratings[k] - ds->residuals[k];
    return predict_host(m, ds->user_idxs, ds->item_idxs, ds->dates, off.data(), ds->n_ratings, out, 0);
}

int tsvd_calc_rmse(const tsvd_model* m, const tsvd_dataset_view* ds, double* out) {
    if (!m || !ds || !out) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (!ds->residuals) throw Error(TSVD_ERR_INVALID, "calc_rmse needs residuals");
        const uint64_t n = ds->n_ratings;
        check_rows(m, ds->user_idxs, ds->item_idxs, n);
        use_device(m);
        cudaStream_t st = m->stream;
        RowStage rs(m, 3 * RowStage::slot(n * 4) + RowStage::slot(n * 2) + RowStage::slot(n));
        const int32_t* du = rs.put(ds->user_idxs, n, st);
        const int32_t* di = rs.put(ds->item_idxs, n, st);
        const int16_t* dd = rs.put(ds->dates, n, st);
        const float* dr = rs.put(ds->residuals, n, st);
        const int8_t* dt = rs.put(ds->is_test, n, st);
        double sse = 0.0, cnt = 0.0;
        tsvd::sse_device(m, du, di, dd, dr, dt, n, &sse, &cnt);
        *out = std::sqrt(sse / cnt);
    });
}

int tsvd_param_nbytes(const tsvd_model* m, const char* name, uint64_t* out) {
    if (!m || !name || !out) return TSVD_ERR_INVALID;
    return guarded(m, [&] {
        std::string n(name);
        if (n == "gbias") { *out = 4; return; }
        if (n == "thresholds" && m->cfg.has_ordinal_head) { *out = 16; return; }
        ParamRef r;
        if (!find_param(m, n, r)) throw Error(TSVD_ERR_INVALID, "unknown or unavailable parameter " + n);
        *out = r.rows * r.cols * 4;
    });
}

int tsvd_get_param(const tsvd_model* m, const char* name, void* dst, uint64_t nbytes) {
    if (!m || !name || !dst) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        std::string n(name);
        use_device(m);
        if (n == "gbias") {
            if (nbytes != 4) throw Error(TSVD_ERR_INVALID, "gbias is 4 bytes");
            std::memcpy(dst, &m->d.gbias, 4);
            return;
        }
        if (n == "thresholds") {
            if (!m->cfg.has_ordinal_head) throw Error(TSVD_ERR_INVALID, "the model has no ordinal head");
            if (nbytes != 16) throw Error(TSVD_ERR_INVALID, "thresholds are 16 bytes");
            std::memcpy(dst, m->h_thresholds, 16);
            return;
        }
        ParamRef r;
        if (!find_param(m, n, r)) throw Error(TSVD_ERR_INVALID, "unknown or unavailable parameter " + n);
        if (nbytes != r.rows * r.cols * 4) throw Error(TSVD_ERR_INVALID, "size mismatch for " + n);
        if (nbytes == 0) return;  // n_feat = 0: feature tables have no columns
        TSVD_CUDA(cudaMemcpy2DAsync(dst, r.cols * 4, r.dev, r.stride * 4, r.cols * 4, r.rows, cudaMemcpyDeviceToHost,
                                    m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int tsvd_set_param(tsvd_model* m, const char* name, const void* src, uint64_t nbytes) {
    if (!m || !name || !src) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        std::string n(name);
        use_device(m);
        if (n == "gbias") {
            if (nbytes != 4) throw Error(TSVD_ERR_INVALID, "gbias is 4 bytes");
            std::memcpy(&m->d.gbias, src, 4);
            return;
        }
        if (n == "tu_mean") throw Error(TSVD_ERR_INVALID, "tu_mean is derived from the data and fixed at create");
        ParamRef r;
        if (!find_param(m, n, r)) throw Error(TSVD_ERR_INVALID, "unknown or unavailable parameter " + n);
        if (nbytes != r.rows * r.cols * 4) throw Error(TSVD_ERR_INVALID, "size mismatch for " + n);
        if (nbytes == 0) return;
        TSVD_CUDA(cudaMemcpy2DAsync(r.dev, r.stride * 4, src, r.cols * 4, r.cols * 4, r.rows, cudaMemcpyHostToDevice,
                                    m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
        if (n == "yfeat" || n == "ybias" || n == "ycache" || n == "ycache_bias") m->ycache_valid = false;
    });
}

int tsvd_copy_rows(tsvd_model* m, const char* name, uint64_t row_lo, uint64_t row_hi, void* d_buf,
                   int32_t to_model) {
    if (!m || !name) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        std::string n(name);
        ParamRef r;
        if (!find_param(m, n, r)) throw Error(TSVD_ERR_INVALID, "unknown parameter " + n);
        // vectors ([n] tables) are one row of n columns: index them by element
        if (r.rows == 1) {
            r.rows = r.cols;
            r.cols = 1;
            r.stride = 1;
        }
        if (row_lo > row_hi || row_hi > r.rows) throw Error(TSVD_ERR_INVALID, "row range out of bounds for " + n);
        const uint64_t rows = row_hi - row_lo;
        if (rows == 0 || r.cols == 0) return;
        if (!d_buf) throw Error(TSVD_ERR_INVALID, "null device buffer");
        use_device(m);
        float* tab = r.dev + row_lo * r.stride;
        if (to_model)
            TSVD_CUDA(cudaMemcpy2DAsync(tab, r.stride * 4, d_buf, r.cols * 4, r.cols * 4, rows, cudaMemcpyDeviceToDevice,
                                        m->stream));
        else
            TSVD_CUDA(cudaMemcpy2DAsync(d_buf, r.cols * 4, tab, r.stride * 4, r.cols * 4, rows, cudaMemcpyDeviceToDevice,
                                        m->stream));
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
        if (to_model && (n == "yfeat" || n == "ybias")) m->ycache_valid = false;
    });
}

int tsvd_row_width(const tsvd_model* m, uint32_t* out) {
    if (!m || !out) return TSVD_ERR_INVALID;
    *out = m->d.Fs;
    return TSVD_OK;
}

int tsvd_user_day_range(const tsvd_model* m, uint32_t u_lo, uint32_t u_hi, uint64_t* ud_lo, uint64_t* ud_hi) {
    if (!m || !ud_lo || !ud_hi) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (u_lo > u_hi || u_hi > m->d.n_users) throw Error(TSVD_ERR_INVALID, "user range out of bounds");
        tsvd_model* mm = const_cast<tsvd_model*>(m);
        if (mm->h_ud_start.empty()) {
            use_device(m);
            mm->h_ud_start.resize((size_t)m->d.n_users + 1);
            TSVD_CUDA(cudaMemcpy(mm->h_ud_start.data(), m->d.ud_start, mm->h_ud_start.size() * 8,
                                 cudaMemcpyDeviceToHost));
        }
        *ud_lo = mm->h_ud_start[u_lo];
        *ud_hi = mm->h_ud_start[u_hi];
    });
}

int tsvd_rebuild_ycache(tsvd_model* m) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        use_device(m);
        tsvd::rebuild_ycache(m);
        tsvd::rebuild_ycache_day(m);
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int tsvd_set_user_order(tsvd_model* m, uint64_t epoch, const uint32_t* perm, uint64_t n) {
    if (!m || !perm) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (n != m->d.n_users) throw Error(TSVD_ERR_INVALID, "permutation length must equal n_users");
        std::vector<uint8_t> seen(n, 0);
        for (uint64_t k = 0; k < n; ++k) {
            if (perm[k] >= n || seen[perm[k]]) throw Error(TSVD_ERR_INVALID, "not a permutation of 0..n_users-1");
            seen[perm[k]] = 1;
        }
        m->injected_order[epoch].assign(perm, perm + n);
    });
}

int tsvd_get_user_order(const tsvd_model* m, uint64_t epoch, uint32_t* perm, uint64_t n) {
    if (!m || !perm) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        if (n != m->d.n_users) throw Error(TSVD_ERR_INVALID, "permutation length must equal n_users");
        auto it = m->injected_order.find(epoch);
        std::vector<uint32_t> o = it != m->injected_order.end()
                                      ? it->second
                                      : tsvd::user_order(n, m->cfg.shuffle_users != 0, m->cfg.seed, epoch);
        std::memcpy(perm, o.data(), n * 4);
    });
}

int tsvd_user_order_for_seed(uint64_t n, int32_t shuffle, uint64_t seed, uint64_t epoch, uint32_t* perm) {
    if (!perm && n) return TSVD_ERR_INVALID;
    return guarded(nullptr, [&] {
        std::vector<uint32_t> o = tsvd::user_order(n, shuffle != 0, seed, epoch);
        if (n) std::memcpy(perm, o.data(), n * 4);
    });
}

int tsvd_normal_stream(uint64_t seed, float sigma, uint64_t n, float* out) {
    if (!out && n) return TSVD_ERR_INVALID;
    return guarded(nullptr, [&] {
        tsvd::ChaCha12Stream g(seed);
        tsvd::fill_normal_rows(g, sigma, 1, n, out, n);
    });
}

int tsvd_set_stream(tsvd_model* m, void* stream) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    m->stream = stream ? (cudaStream_t)stream : m->own_stream;
    return TSVD_OK;
}

int tsvd_synchronize(const tsvd_model* m) {
    if (!m) return TSVD_ERR_INVALID;
    return guarded(m, [&] {
        use_device(m);
        TSVD_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int tsvd_set_profiling(tsvd_model* m, int32_t enabled) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    m->profiling = enabled != 0;
    return TSVD_OK;
}

int tsvd_kernel_stats(const tsvd_model* mc, const char* kernel, uint64_t* launches, double* total_ms) {
    if (!mc || !kernel) return TSVD_ERR_INVALID;
    tsvd_model* m = const_cast<tsvd_model*>(mc);
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        use_device(m);
        tsvd::drain_stats(m);
        auto it = m->stats.find(kernel);
        if (launches) *launches = it == m->stats.end() ? 0 : it->second.launches;
        if (total_ms) *total_ms = it == m->stats.end() ? 0.0 : it->second.total_ms;
    });
}

int tsvd_reset_kernel_stats(tsvd_model* m) {
    if (!m) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(m->mu);
    return guarded(m, [&] {
        use_device(m);
        tsvd::drain_stats(m);
        m->stats.clear();
        m->launches = 0;
    });
}

int tsvd_launch_count(const tsvd_model* m, uint64_t* out) {
    if (!m || !out) return TSVD_ERR_INVALID;
    *out = m->launches;
    return TSVD_OK;
}

}  // extern "C"
