// Batched form: several tsvdx4 variants (different factor sizes, learning
// rates, regularisers) trained together over one device copy of the data.
//
// Hogwild variants: every epoch is one persistent launch over (variant, user)
// work units plus one batched ycache rebuild, captured once as a CUDA graph
// and replayed. Each variant runs its own Hogwild epoch (its own get_users
// order, src/lib.rs:486-494); units of the same position in the variants'
// orders are adjacent, and users with many ratings are moved to the front so
// the longest serial chains start first. The prefetch depth of the Hogwild
// ring is chosen per feature width by an autotuner that times candidate depths
// on throwaway copies of the parameters.
//
// Stratified variants (the deterministic schedule, src/tsvdx4p.rs:815-822):
// every variant's epoch runs on its own stream, forked from and joined back
// to the group's stream, and the whole epoch of all variants is captured once
// as one CUDA graph. A variant's item stratum is bounded by the serial chains
// of its most-rated items, which hold a few SMs; the other variants' strata
// fill the rest of the GPU meanwhile. The autotuner picks, per feature width,
// which items run as whole-CTA tiles (rounds of 32 ratings solved together on
// the tensor cores) and which run one warp each, by timing candidate
// thresholds on throwaway copies.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "rand_stream.hpp"
#include "tsvd_epoch.cuh"

using tsvd::Error;

struct tsvd_group {
    std::vector<tsvd_model*> models;  // models[0] owns the dataset buffers
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string err;
    tsvd::DevMem d_states, d_params, d_units, d_counter;
    uint32_t* h_units = nullptr;  // pinned
    tsvd::DeviceState* h_states = nullptr;  // pinned
    tsvd::EpochParams* h_params = nullptr;  // pinned
    uint32_t n_units = 0;
    uint32_t ring_floats = 0;
    uint32_t heavy_min = 0;  // ratings from which a user is scheduled first
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_graph = true;
    bool stratified = false;
    std::vector<cudaEvent_t> fork, join;  // per variant (stratified)
    uint64_t epochs_run = 0;
    uint64_t launches = 0;
    double last_epoch_ms = 0.0;
};

namespace tsvd {
void setup_params(tsvd_model* m);
}

namespace {

thread_local std::string g_group_err;

template <class F>
int gguard(tsvd_group* g, F&& f) {
    try {
        f();
        return TSVD_OK;
    } catch (const Error& e) {
        if (g) g->err = e.what();
        g_group_err = e.what();
        return e.status;
    } catch (const std::exception& e) {
        if (g) g->err = e.what();
        g_group_err = e.what();
        return TSVD_ERR_INVALID;
    }
}

// A variant sharing models[0]'s dataset buffers; only parameters are new.
tsvd_model* make_variant(const tsvd_model* base, const tsvd_config& cfg) {
    tsvd_model* m = new tsvd_model();
    m->cfg = cfg;
    m->opts = base->opts;
    m->device = base->device;
    TSVD_CUDA(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking));
    m->stream = m->own_stream;
    m->d = base->d;  // dataset part; parameter pointers are replaced below
    m->d.F = (uint32_t)cfg.n_feat;
    m->d.Fs = (uint32_t)((cfg.n_feat + 31) / 32 * 32);
    m->h_user_cnt = base->h_user_cnt;
    tsvd::setup_params(m);
    return m;
}

void check_compatible(const tsvd_config& a, const tsvd_config& b) {
    if (a.n_time_bins != b.n_time_bins || a.n_freq_bins != b.n_freq_bins || a.beta != b.beta ||
        a.low_memory != b.low_memory || a.full_su != b.full_su || a.has_ordinal_head != b.has_ordinal_head)
        throw Error(TSVD_ERR_INVALID,
                    "variants of a group must share n_time_bins, n_freq_bins, beta, low_memory and full_su");
    if (b.n_feat < 1 || b.n_feat > 256) throw Error(TSVD_ERR_UNSUPPORTED, "n_feat must be in 1..256");
}

uint32_t ring_floats_for(const std::vector<tsvd_model*>& ms) {
    uint32_t r = 0;
    for (auto* m : ms) {
        const uint32_t st = tsvd::make_params(m).stages;
        r = std::max<uint32_t>(r, tsvd::hog_ring_floats(st, m->d.Fs));
    }
    return r;
}

void upload_tables(tsvd_group* g) {
    const uint32_t n = (uint32_t)g->models.size();
    for (uint32_t k = 0; k < n; ++k) {
        g->h_states[k] = g->models[k]->d;
        g->h_params[k] = tsvd::make_params(g->models[k]);
        g->h_params[k].stages = g->models[k]->stages;
    }
}

// Units for one epoch: each variant's user order, interleaved by position,
// users without training ratings dropped, heavy users first (stable).
void build_units(tsvd_group* g, uint64_t epoch) {
    const uint32_t n = (uint32_t)g->models.size();
    const uint32_t U = g->models[0]->d.n_users;
    const std::vector<uint32_t>& cnt = g->models[0]->h_user_cnt;
    std::vector<std::vector<uint32_t>> orders(n);
    for (uint32_t k = 0; k < n; ++k) {
        const tsvd_model* m = g->models[k];
        auto it = m->injected_order.find(epoch);
        orders[k] = it != m->injected_order.end() ? it->second
                                                  : tsvd::user_order(U, m->cfg.shuffle_users != 0, m->cfg.seed, epoch);
    }
    uint32_t w = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (uint32_t j = 0; j < U; ++j)
            for (uint32_t k = 0; k < n; ++k) {
                const uint32_t u = orders[k][j];
                const uint32_t c = cnt[u];
                if (c == 0) continue;
                const bool heavy = c >= g->heavy_min;
                if ((pass == 0) == heavy) g->h_units[w++] = (k << 24) | u;
            }
    g->n_units = w;
}

void enqueue_epoch(tsvd_group* g) {
    const uint32_t n = (uint32_t)g->models.size();
    cudaStream_t st = g->stream;
    const uint32_t U = g->models[0]->d.n_users;
    // n_units is the same every epoch (the same users have ratings), so a
    // captured graph stays valid; only the pinned buffers' contents change.
    TSVD_CUDA(cudaMemcpyAsync(g->d_units.p, g->h_units, (size_t)g->n_units * 4, cudaMemcpyHostToDevice, st));
    TSVD_CUDA(cudaMemcpyAsync(g->d_states.p, g->h_states, n * sizeof(tsvd::DeviceState), cudaMemcpyHostToDevice, st));
    TSVD_CUDA(cudaMemcpyAsync(g->d_params.p, g->h_params, n * sizeof(tsvd::EpochParams), cudaMemcpyHostToDevice, st));
    TSVD_CUDA(cudaMemsetAsync(g->d_counter.p, 0, 16, st));
    tsvd::launch_hog_batched(st, g->d_states.as<tsvd::DeviceState>(), g->d_params.as<tsvd::EpochParams>(),
                             g->d_units.as<uint32_t>(), g->n_units, g->ring_floats, g->d_counter.as<uint32_t>());
    tsvd::launch_rebuild_batched(st, g->d_states.as<tsvd::DeviceState>(), n, U);
}

// Every variant's stratified epoch on its own stream: all forked from one
// point of the group's stream, all joined back after every variant's epoch is
// enqueued, so the variants' kernels run concurrently.
void enqueue_strat_epoch(tsvd_group* g, uint64_t epoch) {
    TSVD_CUDA(cudaEventRecord(g->fork[0], g->stream));
    for (size_t k = 0; k < g->models.size(); ++k) {
        tsvd_model* m = g->models[k];
        TSVD_CUDA(cudaStreamWaitEvent(m->stream, g->fork[0], 0));
        tsvd::run_epoch(m, epoch);
        TSVD_CUDA(cudaEventRecord(g->join[k], m->stream));
    }
    for (size_t k = 0; k < g->models.size(); ++k) TSVD_CUDA(cudaStreamWaitEvent(g->stream, g->join[k], 0));
}

void drop_graph(tsvd_group* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->exec = nullptr;
    g->graph = nullptr;
}

// One epoch of stratified variants. The reset epoch of any variant (which
// zeroes that variant's user factors first), the first epoch, and runs with
// the ordinal head (whose epoch end waits on the host) or with kernel
// profiling are launched directly; the others replay one captured graph.
void strat_group_epoch(tsvd_group* g, uint64_t epoch) {
    bool direct = !g->use_graph || g->epochs_run == 0;
    for (auto* m : g->models)
        direct = direct || epoch == m->cfg.reset_u_epoch || m->cfg.has_ordinal_head || m->profiling;
    if (direct) {
        enqueue_strat_epoch(g, epoch);
        return;
    }
    if (!g->exec) {
        TSVD_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_strat_epoch(g, epoch);
        } catch (...) {
            cudaGraph_t dropped = nullptr;
            cudaStreamEndCapture(g->stream, &dropped);
            if (dropped) cudaGraphDestroy(dropped);
            throw;
        }
        TSVD_CUDA(cudaStreamEndCapture(g->stream, &g->graph));
        TSVD_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
    }
    TSVD_CUDA(cudaGraphLaunch(g->exec, g->stream));
}

// Per feature width, the whole-CTA threshold of the item stratum that runs a
// stratified epoch fastest (CUDA events, best of two after a warm-up), timed
// on a throwaway variant with fresh parameters.
void strat_autotune(tsvd_group* g, int32_t* chosen) {
    tsvd_model* m0 = g->models[0];
    const uint32_t cands[] = {0xffffffffu, 65536u, 32768u, 16384u, 8192u, 4096u};
    std::vector<uint32_t> best_for(9, m0->d.heavy_min);
    for (uint32_t vpl = 1; vpl <= 8; ++vpl) {
        const tsvd_model* rep = nullptr;
        for (auto* m : g->models)
            if (m->d.Fs / 32 == vpl) {
                rep = m;
                break;
            }
        if (!rep) continue;
        std::unique_ptr<tsvd_model, void (*)(tsvd_model*)> tmp(make_variant(m0, rep->cfg), tsvd_destroy);
        const uint64_t ep = rep->cfg.reset_u_epoch == 1000000 ? 1000001 : 1000000;
        double best = 1e30;
        for (uint32_t thr : cands) {
            tmp->d.heavy_min = thr;
            double t_best = 1e30;
            for (int rep_i = 0; rep_i < 3; ++rep_i) {
                cudaEvent_t e0, e1;
                TSVD_CUDA(cudaEventCreate(&e0));
                TSVD_CUDA(cudaEventCreate(&e1));
                TSVD_CUDA(cudaEventRecord(e0, tmp->stream));
                tsvd::run_epoch(tmp.get(), ep);
                TSVD_CUDA(cudaEventRecord(e1, tmp->stream));
                TSVD_CUDA(cudaStreamSynchronize(tmp->stream));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                if (rep_i > 0) t_best = std::min<double>(t_best, ms);  // the first run warms up
            }
            if (t_best < best) {
                best = t_best;
                best_for[vpl] = thr;
            }
        }
    }
    for (size_t k = 0; k < g->models.size(); ++k) {
        tsvd_model* m = g->models[k];
        m->d.heavy_min = best_for[m->d.Fs / 32];
        if (chosen) chosen[k] = (int32_t)std::min<uint32_t>(m->d.heavy_min, 0x7fffffffu);
    }
    drop_graph(g);  // the captured graph baked in the old thresholds
}

}  // namespace

extern "C" {

int tsvd_group_create(const tsvd_config* cfgs, uint32_t n_models, const tsvd_gpu_options* opts,
                      const tsvd_dataset_view* tr, const tsvd_dataset_view* pr, tsvd_group** out) {
    if (!out) return TSVD_ERR_INVALID;
    *out = nullptr;
    tsvd_group* g = new tsvd_group();
    int rc = gguard(g, [&] {
        if (!cfgs || n_models == 0 || n_models > 255) throw Error(TSVD_ERR_INVALID, "need 1..255 variants");
        tsvd_gpu_options o{};
        if (opts) o = *opts;
        else o.nsvd_norm_exp = 1.0f;
        if ((o.schedule != TSVD_SCHED_HOGWILD && o.schedule != TSVD_SCHED_STRATIFIED) ||
            o.precision != TSVD_PREC_FP32)
            throw Error(TSVD_ERR_UNSUPPORTED, "the batched form runs Hogwild or stratified epochs in FP32");
        for (int k = 0; k < 5; ++k)
            if (o.seq_epochs[k] != 0) throw Error(TSVD_ERR_UNSUPPORTED, "the batched form has no seq_epochs");
        g->stratified = o.schedule == TSVD_SCHED_STRATIFIED;
        for (uint32_t k = 1; k < n_models; ++k) check_compatible(cfgs[0], cfgs[k]);
        tsvd_model* m0 = nullptr;
        int r0 = tsvd_create(&cfgs[0], &o, tr, pr, &m0);
        if (r0 != TSVD_OK) throw Error(r0, tsvd_last_global_error());
        g->models.push_back(m0);
        g->device = m0->device;
        TSVD_CUDA(cudaSetDevice(g->device));
        for (uint32_t k = 1; k < n_models; ++k) g->models.push_back(make_variant(m0, cfgs[k]));
        for (auto* m : g->models) m->stages = 4;
        TSVD_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        const uint32_t U = m0->d.n_users;
        g->d_units.alloc((size_t)n_models * U * 4);
        g->d_states.alloc(n_models * sizeof(tsvd::DeviceState));
        g->d_params.alloc(n_models * sizeof(tsvd::EpochParams));
        g->d_counter.alloc(16);
        TSVD_CUDA(cudaMallocHost((void**)&g->h_units, (size_t)n_models * U * 4));
        TSVD_CUDA(cudaMallocHost((void**)&g->h_states, n_models * sizeof(tsvd::DeviceState)));
        TSVD_CUDA(cudaMallocHost((void**)&g->h_params, n_models * sizeof(tsvd::EpochParams)));
        const double mean = (double)m0->d.n_train / std::max<uint32_t>(1, U);
        g->heavy_min = (uint32_t)std::max(64.0, 8.0 * mean);
        g->ring_floats = ring_floats_for(g->models);
        if (g->stratified) {
            g->fork.resize(n_models, nullptr);
            g->join.resize(n_models, nullptr);
            for (uint32_t k = 0; k < n_models; ++k) {
                TSVD_CUDA(cudaEventCreateWithFlags(&g->fork[k], cudaEventDisableTiming));
                TSVD_CUDA(cudaEventCreateWithFlags(&g->join[k], cudaEventDisableTiming));
            }
        }
    });
    if (rc != TSVD_OK) {
        tsvd_group_destroy(g);
        return rc;
    }
    *out = g;
    return TSVD_OK;
}

void tsvd_group_destroy(tsvd_group* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (cudaEvent_t e : g->fork)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : g->join)
        if (e) cudaEventDestroy(e);
    for (size_t k = g->models.size(); k-- > 1;) tsvd_destroy(g->models[k]);  // variants borrow models[0]'s data
    if (!g->models.empty()) tsvd_destroy(g->models[0]);
    if (g->h_units) cudaFreeHost(g->h_units);
    if (g->h_states) cudaFreeHost(g->h_states);
    if (g->h_params) cudaFreeHost(g->h_params);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

int tsvd_group_size(const tsvd_group* g, uint32_t* out) {
    if (!g || !out) return TSVD_ERR_INVALID;
    *out = (uint32_t)g->models.size();
    return TSVD_OK;
}

int tsvd_group_model(tsvd_group* g, uint32_t k, tsvd_model** out) {
    if (!g || !out || k >= g->models.size()) return TSVD_ERR_INVALID;
    *out = g->models[k];
    return TSVD_OK;
}

int tsvd_group_set_graphs(tsvd_group* g, int32_t enabled) {
    if (!g) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g->mu);
    g->use_graph = enabled != 0;
    return TSVD_OK;
}

int tsvd_group_fit_epoch(tsvd_group* g, uint64_t epoch) {
    if (!g) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g->mu);
    return gguard(g, [&] {
        if (epoch == 0) throw Error(TSVD_ERR_INVALID, "epochs are 1-based");
        TSVD_CUDA(cudaSetDevice(g->device));
        for (auto* m : g->models) {
            std::lock_guard<std::mutex> mk(m->mu);
            TSVD_CUDA(cudaStreamSynchronize(m->stream));  // no variant work may overlap the epoch
            if (epoch == m->cfg.reset_u_epoch) {
                TSVD_CUDA(cudaMemsetAsync(m->d.ufeat, 0, m->m_ufeat.bytes, g->stream));
                TSVD_CUDA(cudaMemsetAsync(m->d.ufeat2, 0, m->m_ufeat2.bytes, g->stream));
            }
        }
        cudaEvent_t e0, e1;
        TSVD_CUDA(cudaEventCreate(&e0));
        TSVD_CUDA(cudaEventCreate(&e1));
        if (g->stratified) {
            TSVD_CUDA(cudaEventRecord(e0, g->stream));
            try {
                strat_group_epoch(g, epoch);
            } catch (...) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                throw;
            }
            TSVD_CUDA(cudaEventRecord(e1, g->stream));
            TSVD_CUDA(cudaStreamSynchronize(g->stream));
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            g->last_epoch_ms = ms;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            g->epochs_run++;
            return;
        }
        build_units(g, epoch);
        upload_tables(g);
        TSVD_CUDA(cudaEventRecord(e0, g->stream));
        // The first epoch runs uncaptured (it also sets the kernels' launch
        // attributes); later epochs replay one captured graph.
        if (g->use_graph && g->epochs_run > 0) {
            if (!g->exec) {
                TSVD_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    enqueue_epoch(g);
                } catch (...) {
                    cudaGraph_t dropped = nullptr;
                    cudaStreamEndCapture(g->stream, &dropped);
                    if (dropped) cudaGraphDestroy(dropped);
                    throw;
                }
                TSVD_CUDA(cudaStreamEndCapture(g->stream, &g->graph));
                TSVD_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
            }
            TSVD_CUDA(cudaGraphLaunch(g->exec, g->stream));
        } else {
            enqueue_epoch(g);
        }
        TSVD_CUDA(cudaEventRecord(e1, g->stream));
        TSVD_CUDA(cudaStreamSynchronize(g->stream));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        g->last_epoch_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        g->launches += 2;
        g->epochs_run++;
        for (auto* m : g->models) m->ycache_valid = true;
    });
}

int tsvd_group_last_epoch_ms(const tsvd_group* g, double* out) {
    if (!g || !out) return TSVD_ERR_INVALID;
    *out = g->last_epoch_ms;
    return TSVD_OK;
}

// Times the candidate ring depths {2, 3, 4} for each feature width present,
// on throwaway parameter copies (the group's own parameters are not touched),
// over the units of the `sample_users` heaviest users, and keeps the fastest.
int tsvd_group_autotune(tsvd_group* g, uint32_t sample_users, int32_t* chosen_stages) {
    if (!g) return TSVD_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g->mu);
    return gguard(g, [&] {
        TSVD_CUDA(cudaSetDevice(g->device));
        if (g->stratified) {
            strat_autotune(g, chosen_stages);
            return;
        }
        tsvd_model* m0 = g->models[0];
        const uint32_t U = m0->d.n_users;
        std::vector<uint32_t> users(U);
        for (uint32_t u = 0; u < U; ++u) users[u] = u;
        std::stable_sort(users.begin(), users.end(),
                         [&](uint32_t a, uint32_t b) { return m0->h_user_cnt[a] > m0->h_user_cnt[b]; });
        const uint32_t ns = std::min<uint32_t>(std::max<uint32_t>(sample_users, 1), U);
        std::vector<int> width_best(9, 4);
        tsvd::DevMem st_buf, pa_buf, un_buf, cnt_buf;
        st_buf.alloc(sizeof(tsvd::DeviceState));
        pa_buf.alloc(sizeof(tsvd::EpochParams));
        un_buf.alloc((size_t)ns * 4);
        cnt_buf.alloc(16);
        std::vector<uint32_t> units(ns);
        for (uint32_t j = 0; j < ns; ++j) units[j] = users[j];  // variant slot 0
        TSVD_CUDA(cudaMemcpy(un_buf.p, units.data(), ns * 4, cudaMemcpyHostToDevice));
        for (uint32_t vpl = 1; vpl <= 8; ++vpl) {
            const tsvd_model* rep = nullptr;
            for (auto* m : g->models)
                if (m->d.Fs / 32 == vpl) {
                    rep = m;
                    break;
                }
            if (!rep) continue;
            std::unique_ptr<tsvd_model, void (*)(tsvd_model*)> tmp(make_variant(m0, rep->cfg), tsvd_destroy);
            double best = 1e30;
            for (int stages = 2; stages <= 4; ++stages) {
                tsvd::EpochParams p = tsvd::make_params(tmp.get());
                p.stages = stages;
                TSVD_CUDA(cudaMemcpy(st_buf.p, &tmp->d, sizeof(tsvd::DeviceState), cudaMemcpyHostToDevice));
                TSVD_CUDA(cudaMemcpy(pa_buf.p, &p, sizeof(p), cudaMemcpyHostToDevice));
                double t_best = 1e30;
                for (int rep_i = 0; rep_i < 3; ++rep_i) {
                    TSVD_CUDA(cudaMemsetAsync(cnt_buf.p, 0, 16, g->stream));
                    cudaEvent_t e0, e1;
                    TSVD_CUDA(cudaEventCreate(&e0));
                    TSVD_CUDA(cudaEventCreate(&e1));
                    TSVD_CUDA(cudaEventRecord(e0, g->stream));
                    tsvd::launch_hog_batched(g->stream, st_buf.as<tsvd::DeviceState>(),
                                             pa_buf.as<tsvd::EpochParams>(), un_buf.as<uint32_t>(), ns,
                                             tsvd::hog_ring_floats(stages, tmp->d.Fs),
                                             cnt_buf.as<uint32_t>());
                    TSVD_CUDA(cudaEventRecord(e1, g->stream));
                    TSVD_CUDA(cudaStreamSynchronize(g->stream));
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    if (rep_i > 0) t_best = std::min<double>(t_best, ms);  // first run warms up
                }
                if (t_best < best) {
                    best = t_best;
                    width_best[vpl] = stages;
                }
            }
        }
        for (size_t k = 0; k < g->models.size(); ++k) {
            g->models[k]->stages = width_best[g->models[k]->d.Fs / 32];
            if (chosen_stages) chosen_stages[k] = g->models[k]->stages;
        }
        g->ring_floats = 0;
        for (auto* m : g->models)
            g->ring_floats = std::max<uint32_t>(g->ring_floats, tsvd::hog_ring_floats(m->stages, m->d.Fs));
        if (g->exec) {  // the captured graph baked in the old ring size
            cudaGraphExecDestroy(g->exec);
            cudaGraphDestroy(g->graph);
            g->exec = nullptr;
            g->graph = nullptr;
        }
    });
}

const char* tsvd_group_last_error(const tsvd_group* g) { return g ? g->err.c_str() : g_group_err.c_str(); }

}  // extern "C"
