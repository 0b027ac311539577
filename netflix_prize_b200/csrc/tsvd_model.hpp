// Internal state of a tsvd_model: device-resident dataset, precomputed
// per-rating records, parameter tables and scratch. Shared by the ABI,
// setup and kernel translation units. Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tsvdx4_cuda.h"

namespace tsvd {

// Error carrying a tsvd_status.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define TSVD_CUDA(call)                                                                               \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            throw ::tsvd::Error(e_ == cudaErrorMemoryAllocation ? TSVD_ERR_OOM : TSVD_ERR_CUDA,       \
                                std::string(#call) + ": " + cudaGetErrorString(e_) + " at " __FILE__ \
                                ":" + std::to_string(__LINE__));                                      \
    } while (0)

// Owning device allocation.
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    DevMem(DevMem&& o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevMem& operator=(DevMem&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevMem() { release(); }
    void alloc(size_t b) {
        release();
        if (b == 0) b = 16;
        TSVD_CUDA(cudaMalloc(&p, b));
        bytes = b;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return (T*)p; }
};

// Packed per-rating record, 16 bytes, one coalesced load per rating.
//   key = id (20 bits: item in the user-major stream, user in the item-major
//         stream) | time bin << 20 (6 bits) | frequency bin << 26 (6 bits)
//   res = residual (training target), dev = dev_u(t), ud = (user, day) index
struct __align__(16) Rec {
    uint32_t key;
    float res;
    float dev;
    uint32_t ud;
};
constexpr uint32_t kIdBits = 20, kIdMask = (1u << kIdBits) - 1u;
constexpr uint32_t kChunkUsers = 512;  // ratings per chunk of the by-item split sums
constexpr uint32_t kMaxBins = 64;
// Fixed-point scale of the per-day NSVD1 delta sums: integer adds commute, so
// the sums do not depend on the order the users' day runs finish in.
constexpr double kDydScale = 4294967296.0;  // 2^32

// Kernel arguments for one model (everything a kernel may touch).
struct DeviceState {
    // sizes
    uint32_t n_users, n_items, F, Fs, T, NF;
    uint64_t n_train, n_pr, n_ud;
    int32_t day_range;
    float gbias;
    // dataset
    const Rec* rec;            // [n_train] user-major, rating order
    const uint64_t* user_off;  // [U+1]
    const Rec* irec;           // [n_train] item-major (by-item index order)
    const uint64_t* item_off;  // [I+1]
    const uint32_t* pr_item;   // [n_pr] pr items grouped by user, pr order within user
    const uint64_t* pr_off;    // [U+1]
    const int32_t* user_cnt_tr;  // [U]
    const int32_t* user_cnt_pr;  // [U]
    const int8_t* raw;         // [n_train] raw ratings (ordinal head only)
    const uint64_t* ud_start;  // [U+1]
    const int16_t* ud_date;    // [n_ud]
    const uint32_t* ud_cnt;    // [n_ud]
    const float* tu_mean;      // [U]
    // (user, day) item lists, low_memory = false: per ud, its pr items in pr
    // order, then its training items in training order
    const uint64_t* ud_list_off;   // [n_ud + 1]
    const uint32_t* ud_list_item;  // [n_train + n_pr]
    const uint32_t* ud_pr_cnt;     // [n_ud] pr items at the front of each list
    // parameters (feature rows have stride Fs, zero padded)
    float *ubias, *ibias, *ufeat, *ufeat2, *ifeat, *yfeat, *ycache, *yfeat_day;
    float *alpha_u, *but_bin, *bit_bin, *ybias, *ycache_bias;
    float *ubias_day, *ufeat_day, *ycache_day;
    float *ibias_freq, *ifeat_freq, *cu, *cut;
    float* thresholds;  // [4] ordinal head
    // stratified scratch
    float* g_user;   // [U, Fs] per-user NSVD1 gradient sum / norm
    float* e_user;   // [U]     per-user error sum / norm
    float* pyc;      // [U, Fs] p_u + ycache_u for the item stratum; shares g_user's memory,
                     //         which the delta sums have consumed by then
    float* qe0;      // [I, Fs] q_i + q^f_{i,0}, made before each user stratum (low_memory trains
                     //         frequency bin 0, so the user stratum reads only this sum)
    unsigned long long* dyd_fix;  // [I, Fs] low_memory = false: the epoch's yfeat_day deltas,
                                  //         fixed point (kDydScale), added in any order
    // work lists
    const uint32_t* user_work;  // users in processing order
    const uint32_t* item_work;  // items in processing order
    uint32_t n_item_work;       // entries of item_work the item stratum takes (n_items, or a block's)
    uint32_t* counters;         // [8] dynamic work counters
    // fixed-size chunks of the by-item index (deterministic split reductions)
    uint32_t heavy_min;  // item stratum: items with at least this many ratings take a whole block
    uint32_t n_chunks;
    const uint64_t* chunk_lo;      // [n_chunks + 1] start of each chunk in irec; last = n_train
    const uint32_t* item_chunk0;   // [I+1] first chunk of each item
    float* chunk_part;             // [n_chunks, Fs] partial sums
    float* chunk_epart;            // [n_chunks]
};

struct KernelStat {
    uint64_t launches = 0;
    double total_ms = 0.0;
};

}  // namespace tsvd

struct tsvd_model {
    tsvd_config cfg{};
    tsvd_gpu_options opts{};
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    mutable std::mutex mu;
    mutable std::string err;

    tsvd::DeviceState d{};
    bool ycache_valid = false;  // ycache equals a rebuild from the current yfeat
    int stages = 4;             // Hogwild prefetch ring depth when run in a group
    float h_thresholds[4] = {0, 0, 0, 0};  // ordinal head (host copy)
    uint64_t launches = 0;

    // device allocations
    tsvd::DevMem m_rec, m_user_off, m_irec, m_item_off, m_pr_item, m_pr_off, m_ucnt_tr, m_ucnt_pr, m_raw;
    tsvd::DevMem m_ud_start, m_ud_date, m_ud_cnt, m_tu_mean;
    tsvd::DevMem m_ud_list_off, m_ud_list_item, m_ud_pr_cnt;
    tsvd::DevMem m_ubias, m_ibias, m_ufeat, m_ufeat2, m_ifeat, m_yfeat, m_ycache, m_yfeat_day;
    tsvd::DevMem m_alpha_u, m_but_bin, m_bit_bin, m_ybias, m_ycache_bias;
    tsvd::DevMem m_ubias_day, m_ufeat_day, m_ycache_day, m_ibias_freq, m_ifeat_freq, m_cu, m_cut, m_thresholds;
    tsvd::DevMem m_dyd_fix, m_qe0;
    tsvd::DevMem m_g_user, m_e_user, m_user_work, m_item_work, m_counters;
    // BF16 read copies (precision form)
    tsvd::DevMem m_bf_ifeat, m_bf_qf0, m_bf_yfeat, m_bf_pyc, m_bf_ufeat2;
    tsvd::DevMem m_chunk_lo, m_item_chunk0, m_chunk_part, m_chunk_epart;
    tsvd::DevMem m_perm;          // [U] epoch order upload buffer
    // NSVD1 delta-sum passes: per chunk, the positions where the passes' user
    // blocks start ([n_chunks, passes + 1]), for the block bounds last used
    tsvd::DevMem m_chunk_split, m_split_bounds;
    tsvd::DevMem m_shard_work;    // a sharded run's block work list (users or items)
    tsvd::DevMem m_scratch;       // predict / rmse scratch
    // host-buffer entry points (predict, calc_rmse): their rows' device copies,
    // one buffer grown as needed (the model's mutex serialises the calls)
    mutable tsvd::DevMem m_rows;

    std::vector<uint32_t> h_user_cnt;  // train counts (host copy)
    uint32_t h_max_user_cnt = 0;       // the largest of them (made on first use)
    std::vector<uint32_t> h_split_bounds;  // user-block bounds of the delta-sum passes (m_chunk_split)
    std::vector<uint64_t> h_item_off;  // by-item offsets (host copy, made on first use)
    std::vector<uint64_t> h_ud_start;  // (user, day) offsets per user (host copy, made on first use)
    std::map<uint64_t, std::vector<uint32_t>> injected_order;

    // profiling
    bool profiling = false;
    std::map<std::string, tsvd::KernelStat> stats;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
};

namespace tsvd {

// setup (tsvd_setup.cu)
void setup_model(tsvd_model* m, const tsvd_dataset_view& tr, const tsvd_dataset_view& pr);
void setup_params(tsvd_model* m);
// seeded normal init on the device (tsvd_init.cu)
struct NormalTable {
    float* dst;       // rows x stride floats; columns cols..stride-1 are zeroed
    uint64_t rows;
    uint32_t cols, stride;
    float sigma;
};
void device_normal_tables(const NormalTable* tables, int n_tables, uint64_t seed, cudaStream_t st);
// per-day terms, low_memory = false (tsvd_day.cu)
void day_epoch_pass(tsvd_model* m, const uint32_t* order, bool sequential);
void rebuild_ycache_day(tsvd_model* m);
// epoch drivers (tsvd_epoch.cu)
void run_epoch(tsvd_model* m, uint64_t epoch);
void finish_epoch(tsvd_model* m);  // end-of-epoch steps shared by every schedule
void rebuild_ycache(tsvd_model* m);
// predictions (tsvd_predict.cu)
void predict_device(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day,
                    const float* offset, uint64_t n, float* out, int subscores);
void sse_device(const tsvd_model* m, const int32_t* u, const int32_t* i, const int16_t* day, const float* target,
                const int8_t* is_test, uint64_t n, double* out_sse, double* out_cnt);

// profiling helpers (tsvd_abi.cu)
void prof_begin(tsvd_model* m, const char* name, cudaEvent_t* ev_pair);
void prof_end(tsvd_model* m, const char* name, cudaEvent_t* ev_pair);

// RAII scope that records an event pair around launches when profiling.
struct ProfScope {
    tsvd_model* m;
    const char* name;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ProfScope(tsvd_model* mm, const char* n) : m(mm), name(n) { prof_begin(m, name, ev); }
    ~ProfScope() { prof_end(m, name, ev); }
};

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// The calling thread's last error message, shared by every entry point
// (tsvd_last_global_error); defined in tsvd_abi.cu.
std::string& global_err();

// Runs `f` for an extern "C" entry point: every exception becomes a status and
// a message (on the model and the thread), none escapes the C ABI.
template <class F>
int guarded(const tsvd_model* m, F&& f) {
    try {
        f();
        return TSVD_OK;
    } catch (const Error& e) {
        if (m) m->err = e.what();
        global_err() = e.what();
        return e.status;
    } catch (const std::exception& e) {
        if (m) m->err = e.what();
        global_err() = e.what();
        return TSVD_ERR_INVALID;
    }
}

inline void use_device(const tsvd_model* m) { TSVD_CUDA(cudaSetDevice(m->device)); }

}  // namespace tsvd
