/*
 * tsvdx4_cuda.h -- C ABI of the B200 timeSVD++ (tsvdx4) factorizer.
 *
 * This is the drop-in boundary for the reference's model plugin API,
 * `trait Regressor` (src/lib.rs:616-651), as implemented by `TxModel`
 * (src/tx.rs:457-1116) and driven by `fit2_inner`/`fit` (src/lib.rs:881-996,
 * 764-815). A Rust shim `TxGpuModel: Regressor` binds these symbols one to
 * one.
 *
 * Conventions
 *  - Every entry point returns an int status (TSVD_OK == 0). On failure the
 *    message is available from tsvd_last_error(model) (or
 *    tsvd_last_global_error() when no model exists yet). The reference panics
 *    on the same conditions (unwrap/expect/assert!); the shim turns a nonzero
 *    status back into a panic.
 *  - Host arrays are borrowed for the duration of a call only; everything the
 *    model keeps is copied to device memory. No torch types cross this ABI.
 *  - The training set is a full view (ratings and residuals present). The
 *    pr set is passed as a masked view (raw_ratings = residuals = NULL), as
 *    the reference's MaskedDataset hides held-out targets (src/lib.rs:421-455).
 *  - A model is owned by one host thread for mutating calls (create,
 *    fit_epoch, set_*, destroy); const calls (predict_*, rmse, get_param) may
 *    run concurrently from several host threads, which is what `Regressor:
 *    Sync` requires (src/lib.rs:710-722). Const calls serialise internally.
 */
#ifndef TSVDX4_CUDA_H
#define TSVDX4_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSVD_ABI_VERSION 2

enum tsvd_status {
    TSVD_OK = 0,
    TSVD_ERR_INVALID = 1,     /* bad argument, shape or unsorted input      */
    TSVD_ERR_UNSUPPORTED = 2, /* configuration outside the tsvdx4 path      */
    TSVD_ERR_CUDA = 3,        /* CUDA runtime error (message has details)   */
    TSVD_ERR_NO_DEVICE = 4,   /* no usable sm_100 device                    */
    TSVD_ERR_OOM = 5,         /* device allocation failed                   */
    TSVD_ERR_TIMEOUT = 6      /* a bounded device wait ran out              */
};

/* OrdinalHeadConfig (src/lib.rs:502-507). */
typedef struct tsvd_ordinal_config {
    float th_init[4];
    float th_gap;
    float lr_t;
    float reg_t;
} tsvd_ordinal_config;

/* TxConfig (src/tx.rs:128-204), field for field and in the same order.
 * The tsvdx4 path is tx4 mode: lr_w = lr_c = lr_w_day = lr_c_day = 0 and the
 * w_* multipliers 1 (src/tsvdx4.rs:118-136); create() rejects a nonzero
 * neighbourhood learning rate with TSVD_ERR_UNSUPPORTED. */
typedef struct tsvd_config {
    uint64_t n_feat;
    uint64_t n_epochs;
    uint64_t seed;
    int32_t shuffle_users;
    uint64_t n_time_bins;
    float beta;
    uint64_t n_freq_bins;
    float lr_u, lr_ud, lr_u2, lr_ub, lr_ubd, lr_i, lr_ib, lr_y, lr_yb, lr_yd;
    float lr_tu, lr_ti, lr_ta, lr_ibf, lr_iqf, lr_cu;
    float reg_iqf, reg_cu, reg_u, reg_u2, reg_ud, reg_i, reg_y, reg_yd;
    float sigma_iqf, sigma_u, sigma_i, sigma_y, sigma_yd;
    uint64_t reset_u_epoch;
    uint64_t max_neighbors;
    float lr_w, lr_c, reg_w, reg_c;
    float lr_w_day, lr_c_day, reg_w_day, reg_c_day;
    float w_bias, w_factor, w_nbr;
    int32_t sum_err_bug;
    float lambda1, lambda2;
    int32_t has_ordinal_head; /* Option<OrdinalHeadConfig>: 0 = None */
    tsvd_ordinal_config ordinal_head;
    int32_t save_ifeat;
    int32_t low_memory;
    int32_t full_su;
} tsvd_config;

/* Borrowed view of a Dataset (src/lib.rs:227-242). raw_ratings and residuals
 * are NULL in a masked (pr) view. item_idxs is i32 as in memory (i16 on disk,
 * widened at src/lib.rs:255-256). */
typedef struct tsvd_dataset_view {
    const int32_t* user_idxs;
    const int32_t* user_cnts; /* [n_users] */
    const int32_t* item_idxs;
    const int32_t* item_cnts; /* [n_items], may be NULL */
    const int8_t* raw_ratings;
    const float* residuals;
    const int16_t* dates;
    const int8_t* is_test;
    uint64_t n_users;
    uint64_t n_items;
    uint64_t n_ratings;
} tsvd_dataset_view;

/* Epoch schedules. */
enum tsvd_schedule {
    /* Deterministic stratified schedule, the default: the reference's own
     * parallel schedule (src/tsvdx4p.rs:390-805): a user stratum (users in
     * parallel, item tables frozen, NSVD1 deltas reduced in a fixed order),
     * then an item stratum (items in parallel, user tables frozen). Bitwise
     * reproducible for a given seed; held-out RMSE tracks the sequential
     * reference within 0.001 per epoch at the full Netflix shape. Covers
     * both low_memory settings and the ordinal head with lr_t = 0. */
    TSVD_SCHED_STRATIFIED = 0,
    /* Users in parallel, one warp each, item-side tables updated in place as
     * each rating is processed (the reference's per-rating update order
     * inside a user, src/tx.rs:836-1106); concurrent users race on shared
     * item rows. Not bitwise reproducible run to run, and unstable at the
     * full Netflix shape after about 6 epochs of the lm preset (the most
     * rated items' rows go stale under thousands of concurrent users):
     * opt-in, for short runs and moderate sizes. n_feat <= 256. */
    TSVD_SCHED_HOGWILD = 1,
    /* The reference's sequential pass exactly (src/tx.rs:756-1106): one warp
     * takes the users one after another in get_users order, so every rating
     * sees every earlier update. Slow (one warp on the GPU); for parity runs,
     * small data, lr_t != 0 and the seq_epochs of the stratified schedule. */
    TSVD_SCHED_SEQUENTIAL = 2
};

/* Precision forms (stratified schedule only: its strata read frozen tables).
 * Masters are FP32 in every form; accumulation is FP32; the global mean and
 * the SSE/RMSE reductions are FP64. */
enum tsvd_precision {
    TSVD_PREC_FP32 = 0,         /* all reads FP32                                */
    TSVD_PREC_BF16_READ = 1,    /* BF16 read copies of the item tables q_i,
                                   q^f_i and of y_j, refreshed each stratum      */
    TSVD_PREC_BF16_READ_ALL = 2 /* also BF16 copies of the user rows p_u, p2_u,
                                   ycache_u that the item stratum gathers        */
};

/* Options that have no counterpart in TxConfig. Passing opts = NULL to
 * tsvd_create gives the defaults: stratified, FP32, nsvd_norm_exp 1.0,
 * device 0, no sequential epochs. */
typedef struct tsvd_gpu_options {
    int32_t schedule;        /* enum tsvd_schedule                            */
    int32_t precision;       /* enum tsvd_precision                           */
    float nsvd_norm_exp;     /* stratified: y-delta divisor exponent
                                (Tsvdx4pConfig::nsvd_norm_exp,
                                src/tsvdx4p.rs:176-179): 0 = sum, 0.5 = sqrt,
                                1 = mean                                       */
    int32_t device;          /* CUDA device ordinal                           */
    int32_t warps_per_block; /* 0 = tuned default                             */
    int32_t heavy_item_ratings; /* stratified item stratum: items with at least
                                this many ratings take a whole block (rounds of
                                32 ratings solved together), the others one
                                warp each; 0 = default (32768)                 */
    int32_t seq_epochs[5];   /* stratified: Tsvdx4pConfig::seq_epochs
                                (src/tsvdx4p.rs:181-186,815-822): these
                                1-based epochs run the sequential schedule
                                instead; 0 = unused slot                       */
    int32_t reserved[2];
} tsvd_gpu_options;

typedef struct tsvd_model tsvd_model;

/* ---- lifecycle -------------------------------------------------------- */

/* Regressor::new / TxModel::new (src/tx.rs:460-649): computes tu_mean,
 * day_range, SparseUD, user offsets and gbias, and draws the initial factors
 * from StdRng(seed) in the reference's order (ufeat, ifeat, yfeat,
 * [yfeat_day], ifeat_freq) so a seeded run starts where the reference does.
 * opts may be NULL (defaults). */
int tsvd_create(const tsvd_config* cfg, const tsvd_gpu_options* opts,
                const tsvd_dataset_view* tr, const tsvd_dataset_view* pr_masked,
                tsvd_model** out);
void tsvd_destroy(tsvd_model* m);

/* Regressor::n_epochs (src/lib.rs:626). */
int tsvd_n_epochs(const tsvd_model* m, uint64_t* out);

/* Regressor::fit_epoch (src/lib.rs:631; TxModel at src/tx.rs:734-1115).
 * epoch is 1-based. The data were copied at create(); the reference's tr/pr
 * arguments are therefore not passed again. */
int tsvd_fit_epoch(tsvd_model* m, uint64_t epoch);

/* ---- prediction ------------------------------------------------------- */

/* Regressor::predict (src/tx.rs:713-724) for n rows at once: out[k] =
 * predict(u[k], i[k], day[k]) in residual space. Host pointers. */
int tsvd_predict_batch(const tsvd_model* m, const int32_t* u, const int32_t* i,
                       const int16_t* day, uint64_t n, float* out);

/* Same with device pointers, on the model's stream; no host copies and no
 * host-side row checks. A row whose user index is outside 0..n_users-1 or
 * whose item index is outside 0..n_items-1 reads no table and gets a NaN
 * output. */
int tsvd_predict_batch_device(const tsvd_model* m, const int32_t* d_u,
                              const int32_t* d_i, const int16_t* d_day,
                              uint64_t n, float* d_out);

/* Regressor::n_subscores / subscore_names / predict_subscores
 * (src/tx.rs:651-711): 3 columns [bias, mf, nsvd1], out is row-major [n,3]. */
int tsvd_n_subscores(const tsvd_model* m, uint64_t* out);
const char* tsvd_subscore_name(const tsvd_model* m, uint64_t k);
int tsvd_predict_subscores_batch(const tsvd_model* m, const int32_t* u,
                                 const int32_t* i, const int16_t* day,
                                 uint64_t n, float* out);

/* gen_preds_parallel (src/lib.rs:710-722): out[k] = predict(...) +
 * (raw_ratings[k] - residuals[k]) over a full view. */
int tsvd_gen_preds(const tsvd_model* m, const tsvd_dataset_view* ds, float* out);

/* calc_rmse (src/lib.rs:659-672): FP64 sum of squared errors over the
 * is_test == 0 rows of a full view. */
int tsvd_calc_rmse(const tsvd_model* m, const tsvd_dataset_view* ds, double* out);

/* Allocation-free RMSE over device-resident rows. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they evaluate (memory reserved up front by the process owner, a caching
 * allocator that must not be bypassed, or a latency-sensitive loop that may
 * not call cudaMalloc/cudaFree, which can synchronise the device).
 * Inputs d_u, d_i, d_day, d_target (and d_is_test, which may be NULL) are
 * device arrays of n rows; d_out is a device array of 3 doubles that receives
 * {rmse, sum of squared errors, rows counted} over the is_test == 0 rows.
 * Rows whose user or item index is out of range are never read; if there is
 * any, d_out receives {NaN, NaN, -(number of such rows)} instead.
 * The result equals tsvd_calc_rmse's up to FP64 summation order.
 * It calls no allocator: its scratch is a fixed 512 KiB device array inside
 * the library (held by every GPU that loads it until exit), which limits n to
 * 134,217,728 rows; larger n returns TSVD_ERR_INVALID. The scratch's device
 * address is looked up on the first call on each device, so make that first
 * call before any stream capture. Work is enqueued on the model's stream and
 * not waited for. All calls share the scratch: calls that overlap on the GPU
 * (different streams, no ordering between them) race and give wrong results. */
int tsvd_calc_rmse_device_noalloc(const tsvd_model* m, const int32_t* d_u,
                                  const int32_t* d_i, const int16_t* d_day,
                                  const float* d_target, const int8_t* d_is_test,
                                  uint64_t n, double* d_out);

/* ---- parameters ------------------------------------------------------- */

/* Names: gbias, ubias, ibias, ufeat, ufeat2, ifeat, yfeat, ycache, yfeat_day,
 * tu_mean, alpha_u, but_bin, bit_bin, ybias, ycache_bias, ubias_day,
 * ufeat_day, ycache_day, ibias_freq, ifeat_freq, cu, cut, thresholds.
 * All are f32, row-major, shaped as in TxModel (src/tx.rs:210-272).
 * get copies to host; set copies from host (nbytes must match exactly).
 * Setting yfeat/ybias does not rebuild ycache; call tsvd_rebuild_ycache. */
int tsvd_param_nbytes(const tsvd_model* m, const char* name, uint64_t* out);
int tsvd_get_param(const tsvd_model* m, const char* name, void* dst, uint64_t nbytes);
int tsvd_set_param(tsvd_model* m, const char* name, const void* src, uint64_t nbytes);

/* TxModel::rebuild_ycache (+ _day) (src/tx.rs:391-454). */
int tsvd_rebuild_ycache(tsvd_model* m);

/* Inject the user order of one epoch (a permutation of 0..n_users-1) in
 * place of get_users(n, shuffle, seed, epoch) (src/lib.rs:486-494). */
int tsvd_set_user_order(tsvd_model* m, uint64_t epoch, const uint32_t* perm, uint64_t n);

/* The order get_users would produce for this epoch (rand 0.9 StdRng shuffle). */
int tsvd_get_user_order(const tsvd_model* m, uint64_t epoch, uint32_t* perm, uint64_t n);

/* Standalone seeded streams (no model, no device needed):
 * get_users(n, shuffle, seed, epoch) (src/lib.rs:486-494) and the first n
 * draws of rand_array2(.., &mut StdRng::seed_from_u64(seed), sigma)
 * (src/lib.rs:64-67). */
int tsvd_user_order_for_seed(uint64_t n, int32_t shuffle, uint64_t seed, uint64_t epoch, uint32_t* perm);
int tsvd_normal_stream(uint64_t seed, float sigma, uint64_t n, float* out);

/* ---- sharded runs: one process per GPU --------------------------------- */

/* One stratified epoch split over P processes (one per GPU), users and items
 * in contiguous blocks, each process holding a full model (item tables and
 * NSVD1 tables replicated, every process creating it from the same data and
 * config). The steps of Tsvdx4pModel::fit_epoch (src/tsvdx4p.rs:815-822) with
 * the caller's collectives between them (device buffers, e.g. NCCL):
 *   1. tsvd_shard_user_block(own user block): the user stratum of the block's
 *      users (fit_epoch_user, :390-639) and the block's NSVD1 delta sums per
 *      item (NsvdDelta, :63-80): d_sums [n_items, Fs] floats (Fs = the padded
 *      row width, tsvd_row_width), d_sums_e [n_items]; with low_memory = false
 *      also d_dyd [n_items, Fs] int64, the yfeat_day sums in fixed point;
 *   2. all-reduce (sum) of those three buffers over the processes;
 *   3. all-gather of the user blocks' rows: ufeat, ufeat2, ubias, alpha_u, cu,
 *      but_bin, and over each block's (user, day) range (tsvd_user_day_range)
 *      ubias_day and, with low_memory = false, ufeat_day (tsvd_copy_rows);
 *   4. tsvd_shard_apply(the summed buffers): apply_nsvd_deltas (:341-385) and
 *      the ycache (and ycache_day) rebuild;
 *   5. tsvd_shard_item_block(own item block): fit_epoch_item (:644-762) for
 *      the block's items, then the end-of-epoch steps;
 *   6. all-gather of the item blocks' rows: ifeat, ifeat_freq (rows
 *      i * n_freq_bins ..), ibias, bit_bin, ibias_freq.
 * Every process then holds the same model. Results equal the one-process
 * stratified epoch up to the order of the delta additions. Stratified
 * schedule, FP32 only. No counterpart in the reference beyond the steps
 * cited (its parallel schedule runs on the threads of one host). */
int tsvd_shard_user_block(tsvd_model* m, uint64_t epoch, uint32_t u_lo, uint32_t u_hi,
                          float* d_sums, float* d_sums_e, int64_t* d_dyd);
int tsvd_shard_apply(tsvd_model* m, const float* d_sums, const float* d_sums_e,
                     const int64_t* d_dyd);
int tsvd_shard_item_block(tsvd_model* m, uint32_t i_lo, uint32_t i_hi);
/* Rows row_lo..row_hi-1 of a parameter table (names as for tsvd_get_param;
 * an [n] vector's rows are its elements) to (to_model = 0) or from
 * (to_model = 1) a packed device buffer of (row_hi - row_lo) x columns floats,
 * on the model's stream, waited for. */
int tsvd_copy_rows(tsvd_model* m, const char* name, uint64_t row_lo, uint64_t row_hi,
                   void* d_buf, int32_t to_model);
/* The (user, day) rows [ud_lo, ud_hi) of users u_lo..u_hi-1 (SparseUD,
 * src/tx.rs:21-84: a user's days are contiguous). */
int tsvd_user_day_range(const tsvd_model* m, uint32_t u_lo, uint32_t u_hi,
                        uint64_t* ud_lo, uint64_t* ud_hi);
/* Fs: the padded row width of the feature tables (n_feat rounded up to 32,
 * or to 256 above 256; 32 for n_feat = 0). */
int tsvd_row_width(const tsvd_model* m, uint32_t* out);

/* ---- batched form: several variants in one persistent launch ---------- */

/* A group of variants over one dataset, e.g. the lr/reg/n_feat grid of a
 * hyperparameter search. Each variant is a TxModel (src/tx.rs:457-1116) with
 * its own parameters and Hogwild epochs (its own get_users order); the data
 * are held once. Variants must share n_time_bins, n_freq_bins, beta,
 * low_memory and full_su. opts must select Hogwild / FP32. */
typedef struct tsvd_group tsvd_group;
int tsvd_group_create(const tsvd_config* cfgs, uint32_t n_models,
                      const tsvd_gpu_options* opts, const tsvd_dataset_view* tr,
                      const tsvd_dataset_view* pr_masked, tsvd_group** out);
void tsvd_group_destroy(tsvd_group* g);
int tsvd_group_size(const tsvd_group* g, uint32_t* out);
/* Borrowed model k: predict/rmse/get_param/set_param work on it; it must not
 * be destroyed by the caller and lives as long as the group. */
int tsvd_group_model(tsvd_group* g, uint32_t k, tsvd_model** out);
/* One epoch of every variant: one persistent launch plus one batched ycache
 * rebuild; from the second epoch on they replay one captured CUDA graph. */
int tsvd_group_fit_epoch(tsvd_group* g, uint64_t epoch);
/* 0 = launch directly every epoch (no CUDA graph). */
int tsvd_group_set_graphs(tsvd_group* g, int32_t enabled);
/* Device time of the last group epoch (CUDA events around the launch). */
int tsvd_group_last_epoch_ms(const tsvd_group* g, double* out);
/* Picks the Hogwild prefetch depth (2..4 staged ratings) per feature width by
 * timing each candidate on throwaway parameter copies over the units of the
 * sample_users heaviest users; chosen_stages (n_models ints) may be NULL. */
int tsvd_group_autotune(tsvd_group* g, uint32_t sample_users, int32_t* chosen_stages);
const char* tsvd_group_last_error(const tsvd_group* g);

/* ---- learned warm start: amortised user encoder + fold-in --------------- */

/* No counterpart in the reference. An encoder predicts a user's p_u, b_u and
 * alpha_u from the user's training history (embedding bag over item, rating
 * and time bin, dim 128; MLP 128 -> 512 -> 512 -> f+2 with GELU; BF16
 * tensor-core GEMMs, FP32 accumulation, FP32 master weights, AdamW). Targets
 * are the current factors of model m for the target users, standardised per
 * dimension with statistics of target_users. train_raw is the training set's
 * raw_ratings column (n_train entries, values 1..5). */
typedef struct tsvd_encoder tsvd_encoder;
int tsvd_encoder_create(const tsvd_model* m, const int8_t* train_raw,
                        const uint32_t* target_users, uint64_t n_target,
                        uint64_t seed, float lr, float weight_decay,
                        tsvd_encoder** out);
void tsvd_encoder_destroy(tsvd_encoder* e);
/* One pass over users in mini-batches of `batch` (<= 4096): forward, MSE,
 * backward, AdamW step. */
int tsvd_encoder_train_epoch(tsvd_encoder* e, const uint32_t* users, uint64_t n,
                             uint32_t batch, double* mean_loss);
/* Loss and gradients of one batch (n <= 4096) without an update; gradients
 * are read with tsvd_encoder_get("g.<name>"). */
int tsvd_encoder_loss_grad(tsvd_encoder* e, const uint32_t* users, uint32_t n, double* loss);
/* Standardised outputs [n, f+2] (n <= 4096). */
int tsvd_encoder_forward(tsvd_encoder* e, const uint32_t* users, uint32_t n, float* out);
/* Writes de-standardised predictions of p_u, b_u, alpha_u into model m for
 * `users` and resets their other user state to the standard init. */
int tsvd_encoder_apply(tsvd_encoder* e, tsvd_model* m, const uint32_t* users, uint64_t n);
/* Parameters (or gradients as "g.<name>"): e_item [n_items * 5, 128] (row
 * 5 i + r - 1 for item i rated r), e_rate [5, 128], e_date [T, 128], w1, b1,
 * w2, b2, w3, b3; FP32, matrices [in, out] row-major. */
int tsvd_encoder_get(const tsvd_encoder* e, const char* name, float* dst, uint64_t count);
int tsvd_encoder_set(tsvd_encoder* e, const char* name, const float* src, uint64_t count);
int tsvd_encoder_target_stats(const tsvd_encoder* e, float* mean, float* std_out);
const char* tsvd_encoder_last_error(const tsvd_encoder* e);

/* Fold-in: `passes` user-side SGD passes over `users` with every item-side
 * table frozen -- the user phase of the reference's parallel schedule
 * (src/tsvdx4p.rs:390-639) restricted to those users, without the NSVD1
 * delta step. */
int tsvd_foldin(tsvd_model* m, const uint32_t* users, uint64_t n, uint32_t passes);

/* Standard init of `users`' state (p_u ~ N(0, sigma_u) from StdRng(seed),
 * everything else as TxModel::new sets it), for fold-in baselines. */
int tsvd_reset_users(tsvd_model* m, const uint32_t* users, uint64_t n, uint64_t seed);

/* ---- streams, timing, errors ------------------------------------------ */

/* Launch all work of this model on `stream` (a cudaStream_t); NULL = the
 * model's own stream. */
int tsvd_set_stream(tsvd_model* m, void* stream);
int tsvd_synchronize(const tsvd_model* m);

/* Per-kernel CUDA-event timing, recorded on the launching stream.
 * Enabling adds an event pair around each launch. */
int tsvd_set_profiling(tsvd_model* m, int32_t enabled);
int tsvd_kernel_stats(const tsvd_model* m, const char* kernel, uint64_t* launches,
                      double* total_ms);
int tsvd_reset_kernel_stats(tsvd_model* m);
/* Number of kernels this model has launched since create (or the last
 * reset_kernel_stats). */
int tsvd_launch_count(const tsvd_model* m, uint64_t* out);

const char* tsvd_last_error(const tsvd_model* m);
const char* tsvd_last_global_error(void);
int tsvd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TSVDX4_CUDA_H */
