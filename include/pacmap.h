/*
 * pacmap.h -- C ABI of the B200-native PaCMAP engine (libpacmap_b200.so).
 *
 * Drop-in boundary for beamform/pacmap-rs v0.2.6 (crate `pacmap`). The reference's public API is Rust:
 *   fit_transform(x: ArrayView2<f32>, config: Configuration)
 *       -> Result<(Array2<f32>, Option<Array3<f32>>), PaCMapError>                     src/lib.rs:294-297
 *   knn::find_k_nearest_neighbors(data: ArrayView2<f32>, k: usize)
 *       -> (Array2<u32>, Array2<f32>)                                                   src/knn.rs:137
 * Each entry point below names the reference item it replaces. A Rust (or any FFI) binding wraps these
 * with the reference's types; the Python mirror in pacmap-rs_b200/pacmap_b200 does exactly that.
 *
 * Conventions (as in the reference, src/lib.rs:294-367): synchronous; inputs borrowed; every matrix is
 * row-major and dense; outputs go to caller-owned buffers of the documented size; errors are status
 * codes (the reference's Result), with a thread-local message from pacmap_last_error(). All compute runs
 * on one CUDA device (cfg->device); there is no CPU fallback: without a usable sm_100 device every
 * compute entry point returns PACMAP_ERR_NO_DEVICE. Calls from several host threads are safe; calls on
 * one device are serialised.
 */
#ifndef PACMAP_B200_H
#define PACMAP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PaCMapError (src/lib.rs:870-922) and KnnError (src/knn.rs:196-206), one code per variant, plus the
 * conditions the reference turns into panics or endless loops, and device-side failures. */
typedef enum pacmap_status {
  PACMAP_OK = 0,
  PACMAP_ERR_SAMPLE_SIZE = 1,               /* SampleSize: n <= 1                       lib.rs:875 */
  PACMAP_ERR_INVALID_NN_SHAPE = 2,          /* InvalidNearestNeighborShape              lib.rs:879 */
  PACMAP_ERR_EMPTY_ARRAY_MEAN = 3,          /* EmptyArrayMean                           lib.rs:888 */
  PACMAP_ERR_NORMAL = 4,                    /* Normal (distribution construction)       lib.rs:892 */
  PACMAP_ERR_INVALID_NEIGHBOR_COUNT = 5,    /* InvalidNeighborCount                     lib.rs:896 */
  PACMAP_ERR_INVALID_FAR_POINT_COUNT = 6,   /* InvalidFarPointCount                     lib.rs:900 */
  PACMAP_ERR_EMPTY_ARRAY_MIN_MAX = 7,       /* EmptyArrayMinMax                         lib.rs:904 */
  PACMAP_ERR_ZERO_RANGE = 8,                /* ZeroRange (never raised, as in the ref.) lib.rs:908 */
  PACMAP_ERR_PCA = 9,                       /* Pca                                      lib.rs:912 */
  PACMAP_ERR_KNN_CONSTRUCTION = 10,         /* KnnError::Construction                   knn.rs:200 */
  PACMAP_ERR_KNN_RESERVATION = 11,          /* KnnError::Reservation                    knn.rs:204 */
  PACMAP_ERR_MISSING_TRANSFORM = 12,        /* MissingTransform                         lib.rs:920 */
  PACMAP_ERR_INVALID_ARGUMENT = 20,         /* NULL pointer / bad enum / size overflow               */
  PACMAP_ERR_PAIR_INDEX = 21,               /* a provided pair names a point >= n (the ref. panics)  */
  PACMAP_ERR_SAMPLING = 22,                 /* distinct partners cannot be drawn (the ref. spins)    */
  PACMAP_ERR_UNSUPPORTED = 23,              /* a size beyond a kernel limit                          */
  PACMAP_ERR_MODEL_FILE = 24,               /* a model file cannot be read/written or is damaged     */
  PACMAP_ERR_CUDA = 30,                     /* CUDA runtime error (message has the detail)           */
  PACMAP_ERR_OOM = 31,                      /* device allocation failed                              */
  PACMAP_ERR_NO_DEVICE = 32,                /* no CUDA device of compute capability 10.x             */
  PACMAP_ERR_DEVICE_INVARIANT = 33          /* a kernel's own check failed (index range, timeout)    */
} pacmap_status;

/* Initialization (src/lib.rs:226-239). PCA: the exact principal axes (pacmap-rs_b200/csrc/pca.cu) where
 * the reference calls petal-decomposition's SVD / randomized SVD; with d > 100 the pairs are drawn on
 * the projection onto min(100, n) axes, as the reference does (src/lib.rs:455-480). */
typedef enum pacmap_init_kind {
  PACMAP_INIT_PCA = 0,
  PACMAP_INIT_VALUE = 1,  /* Value(Array2<f32>): init_value, n x embedding_dimensions           */
  PACMAP_INIT_RANDOM = 2  /* Random(Option<u64>): init_has_seed / init_seed                     */
} pacmap_init_kind;

/* PairConfiguration (src/lib.rs:241-267). */
typedef enum pacmap_pair_kind {
  PACMAP_PAIRS_GENERATE = 0,
  PACMAP_PAIRS_NEIGHBORS_PROVIDED = 1,  /* pair_neighbors: (n*k) x 2                               */
  PACMAP_PAIRS_ALL_PROVIDED = 2         /* pair_neighbors, pair_mn, pair_fp: rows x 2 each          */
} pacmap_pair_kind;

/* How the kNN is computed (no reference analogue). Modes 0-3 and 5 return identical exact indices and
 * distances; mode 4 is approximate from approx_threshold rows on. From 32,768 rows the tensor-core modes
 * (0-2) skip the column tiles that provably hold no neighbour of a row block (a triangle-inequality
 * bound through pivot points against a first pass's neighbour-distance bound); mode 5 computes every
 * tile. */
typedef enum pacmap_knn_mode {
  PACMAP_KNN_AUTO = 0,         /* tensor-core filter when the dimension allows it, else SIMT exact   */
  PACMAP_KNN_TENSOR_F16 = 1,   /* tcgen05 FP16 distance GEMM filter + exact FP32 re-rank            */
  PACMAP_KNN_TENSOR_BF16 = 2,  /* tcgen05 BF16 distance GEMM filter + exact FP32 re-rank            */
  PACMAP_KNN_SIMT_EXACT = 3,   /* every distance in the reference's FP32 order on CUDA cores        */
  PACMAP_KNN_APPROX = 4,       /* approximate at n >= approx_threshold (the reference's rule,
                                * src/neighbors.rs:71): each row block searches only the 16 of 256
                                * pivot cells nearest its own; returned distances stay exact. Below
                                * the threshold (or below 16,384 rows, where the SIMT path runs) exact;
                                * pacmap_knn_exact has no threshold: approximate whenever it can be. */
  PACMAP_KNN_TENSOR_F16_FULL = 5  /* as TENSOR_F16 with every column tile computed (no pruning)     */
} pacmap_knn_mode;

/* The distance the pairs are drawn with (no reference analogue: the reference is Euclidean only,
 * README.md:164). ANGULAR divides every preprocessed row by its norm (the reference's f32 distance from
 * the origin; zero rows stay zero), so that Euclidean distances become the angular distance
 * sqrt(2 - 2 cos) of the preprocessed rows; the kNN, sigma scaling and mid-near choices follow it. */
typedef enum pacmap_metric {
  PACMAP_METRIC_EUCLIDEAN = 0,  /* the reference's metric                                            */
  PACMAP_METRIC_ANGULAR = 1
} pacmap_metric;

/* Configuration (src/lib.rs:159-224), field by field, plus the engine's switches at the end.
 * Option<T> fields are a has_ flag plus the value. Pointers are host memory and only read. */
typedef struct pacmap_config {
  uint64_t embedding_dimensions;       /* default 2                                                  */
  int32_t init_kind;                   /* pacmap_init_kind, default PCA (as the reference)          */
  const float* init_value;             /* VALUE: n x embedding_dimensions                           */
  int32_t init_has_seed;               /* RANDOM(Some(seed)) when 1, RANDOM(None) when 0            */
  uint64_t init_seed;
  float mid_near_ratio;                /* default 0.5                                                */
  float far_pair_ratio;                /* default 2.0                                                */
  int32_t has_override_neighbors;      /* override_neighbors: Option<usize>                          */
  uint64_t override_neighbors;
  int32_t has_seed;                    /* seed: Option<u64> (pair sampling)                          */
  uint64_t seed;
  int32_t pair_kind;                   /* pacmap_pair_kind, default GENERATE                        */
  const uint32_t* pair_neighbors;      /* NEIGHBORS_PROVIDED / ALL_PROVIDED                         */
  uint64_t pair_neighbors_rows;
  const uint32_t* pair_mn;             /* ALL_PROVIDED                                               */
  uint64_t pair_mn_rows;
  const uint32_t* pair_fp;             /* ALL_PROVIDED                                               */
  uint64_t pair_fp_rows;
  float learning_rate;                 /* default 1.0                                                */
  uint64_t num_iters[3];               /* default (100, 100, 250)                                    */
  const uint64_t* snapshots;           /* Option<Vec<usize>>: NULL = None                            */
  uint64_t n_snapshots;
  uint64_t approx_threshold;           /* default 8000; used by knn_mode APPROX only (else exact)    */
  /* --- engine switches (no reference analogue) --- */
  int32_t knn_mode;                    /* pacmap_knn_mode, default AUTO                              */
  int32_t device;                      /* CUDA device ordinal, default 0                             */
  float* loss_trace;                   /* optional out: the loss (grad[n,0]) of every iteration      */
  int32_t metric;                      /* pacmap_metric, default EUCLIDEAN                          */
} pacmap_config;

/* Configuration::default() (src/lib.rs:208-224) plus the engine defaults. */
pacmap_config pacmap_config_default(void);

/* fit_transform (src/lib.rs:294-367). x: n x d. out_embedding: n x embedding_dimensions.
 * out_snapshots: n_snapshots x n x embedding_dimensions, or NULL (ignored when cfg->snapshots is NULL).
 * Slot semantics follow src/lib.rs:789-791,830-836: slot 0 starts as the initial embedding; iteration
 * itr (0-based) writes the first slot whose index equals itr + 1. */
pacmap_status pacmap_fit_transform(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                   float* out_embedding, float* out_snapshots);

/* Same as pacmap_fit_transform with x, out_embedding (and out_snapshots) in device memory of
 * cfg->device (no reference analogue: it keeps host<->device copies out of a caller's timing). */
pacmap_status pacmap_fit_transform_device(const float* d_x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                          float* d_out_embedding, float* d_out_snapshots);

/* knn::find_k_nearest_neighbors (src/knn.rs:137-194): exact Euclidean kNN of the rows of x (not
 * preprocessed), self excluded, k' = min(k, n-1) columns in ascending (f32 distance, index) order.
 * out_idx, out_dist: n x k'. n == 0 is a no-op. Distances are the reference's f32 values. */
pacmap_status pacmap_knn_exact(const float* x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode,
                               int32_t device, uint32_t* out_idx, float* out_dist);

/* One shard of pacmap_knn_exact for multi-GPU use (no reference analogue): every rank passes all
 * points and computes the rows of shard `shard` of `n_shards` (the tensor-core path splits its row
 * blocks in its locality order, the SIMT path the rows in order). out_idx, out_dist: n x k' with the
 * shard's rows filled and the others zero; out_owned (n bytes): 1 on the rows filled. The shards of
 * one (x, k, knn_mode) partition the rows, and their union is pacmap_knn_exact's output bit for bit. */
pacmap_status pacmap_knn_exact_shard(const float* x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode,
                                     uint32_t shard, uint32_t n_shards, int32_t device, uint32_t* out_idx,
                                     float* out_dist, uint8_t* out_owned);

/* pacmap_knn_exact_shard with d_x, the outputs and the owned mask in device memory of `device` (no
 * reference analogue): the shard stays on the GPU for a collective assembly (pacmap_b200.knn). The call
 * returns when the shard is complete. */
pacmap_status pacmap_knn_exact_shard_device(const float* d_x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode,
                                            uint32_t shard, uint32_t n_shards, int32_t device, uint32_t* d_out_idx,
                                            float* d_out_dist, uint8_t* d_out_owned);

/* --- stage entry points: the parity harness and callers that run part of the pipeline --- */

/* preprocess_x non-PCA branch (src/lib.rs:485-511): out = (x - min) / max - column mean. x, out: n x d.
 * out_mean: d values (may be NULL). */
pacmap_status pacmap_preprocess(const float* x, uint64_t n, uint64_t d, int32_t device, float* out,
                                float* out_min, float* out_max, float* out_mean);

/* sample_pairs with PairConfiguration::Generate (src/lib.rs:641-648 -> src/neighbors.rs:56-108) on the
 * raw x: preprocessing, exact kNN with k+50 candidates, sigma scaling, reselection, MN and FP sampling.
 * Pair counts come from decide_num_pairs (src/lib.rs:565-597); out_counts receives (k, n_mn, n_fp)
 * where k = min(n_neighbors, n-1). Buffers: out_pnn (n*k x 2), out_pmn (n*n_mn x 2), out_pfp
 * (n*n_fp x 2); any may be NULL to only query the counts. */
pacmap_status pacmap_generate_pairs(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                    uint64_t* out_counts, uint32_t* out_pnn, uint32_t* out_pmn,
                                    uint32_t* out_pfp);

/* generate_pairs steps after the kNN (src/neighbors.rs:79-89, src/sampling.rs:251-286): sigma from the
 * 4th-6th neighbour distances, scaled distances, the k best per row. knn_idx/knn_dist: n x kp.
 * out_pnn: (n*k) x 2. out_sigma (n, may be NULL). */
pacmap_status pacmap_reselect_neighbors(const uint32_t* knn_idx, const float* knn_dist, uint64_t n,
                                        uint64_t kp, uint64_t k, int32_t device, uint32_t* out_pnn,
                                        float* out_sigma);

/* sample_mn_pair_deterministic / sample_fp_pair_deterministic (src/sampling.rs:77-142) on the
 * library's Philox stream. xp: the preprocessed n x d data. out_pmn: (n*n_mn) x 2; out_pfp:
 * (n*n_fp) x 2 given pair_neighbors ((n*k) x 2). Either output may be NULL to skip it. */
pacmap_status pacmap_sample_pairs(const float* xp, uint64_t n, uint64_t d, const uint32_t* pair_neighbors,
                                  uint64_t k, uint64_t n_mn, uint64_t n_fp, uint64_t seed, int32_t device,
                                  uint32_t* out_pmn, uint32_t* out_pfp);

/* The optimiser loop (src/lib.rs:800-837) from an explicit state: iterations [itr_begin, itr_end) of
 * weights -> gradient -> Adam, starting from y, m, v (n x dim each, updated in place). The schedule
 * (num_iters p1, p2) and lr set the weights and the bias-corrected step. out_grad (optional,
 * (n+1) x dim): the gradient of the last iteration, loss at [n, 0]. */
pacmap_status pacmap_optimize_steps(float* y, float* m, float* v, uint64_t n, uint64_t dim,
                                    const uint32_t* pnn, uint64_t n_nn, const uint32_t* pmn, uint64_t n_mn,
                                    const uint32_t* pfp, uint64_t n_fp, float learning_rate, uint64_t p1,
                                    uint64_t p2, uint64_t itr_begin, uint64_t itr_end, int32_t device,
                                    float* out_grad);

/* pacmap_grad (src/gradient.rs:35-74) with explicit weights: out_grad ((n+1) x dim) receives the
 * gradient of every point and the loss at [n, 0]. */
pacmap_status pacmap_gradient(const float* y, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn,
                              const uint32_t* pmn, uint64_t n_mn, const uint32_t* pfp, uint64_t n_fp, float w_nn,
                              float w_mn, float w_fp, int32_t device, float* out_grad);

/* Initialization::Value (src/lib.rs:753-766) applied on the device: (v - mean) * 1e-4 / std. */
pacmap_status pacmap_init_value(const float* v, uint64_t n, uint64_t dim, int32_t device, float* out);

/* Initialization::Random(seed) on the library's Philox stream (N(0,1), Box-Muller). */
pacmap_status pacmap_init_random(uint64_t n, uint64_t dim, uint64_t seed, int32_t device, float* out);

/* --- the learned initialiser (no reference analogue) ---
 * An MLP d -> 512 -> 512 -> dim (ReLU; BF16 weights and activations, FP32 accumulation; every GEMM a
 * tcgen05 kernel) maps preprocessed data x' (the output of pacmap_preprocess) to an embedding, used as
 * Initialization::Value (src/lib.rs:753-766) so that a shortened schedule suffices. Parameters are one
 * flat f32 array: [W1 (512 x d), b1 (512), W2 (512 x 512), b2 (512), W3 (dim x 512), b3 (dim)]. */
uint64_t pacmap_mlp_param_count(uint64_t d, uint64_t dim);
/* Seeded U(-1/sqrt(fan_in), 1/sqrt(fan_in)) initial parameters. */
pacmap_status pacmap_mlp_init(uint64_t d, uint64_t dim, uint64_t seed, float* out_params);
/* AdamW training on (x' rows, target embedding rows; targets are z-scored per dimension), mean squared
 * error, `epochs` passes in shuffled batches of `batch` rows (a multiple of 128). inout_params: the
 * starting parameters, replaced by the trained ones. out_epoch_loss (optional): epochs values. */
pacmap_status pacmap_mlp_train(const float* xp, const float* target, uint64_t n, uint64_t d, uint64_t dim,
                               uint64_t epochs, uint64_t batch, float lr, float weight_decay, uint64_t seed,
                               int32_t device, float* inout_params, float* out_epoch_loss);
/* out (n x dim) = MLP(xp). */
pacmap_status pacmap_mlp_apply(const float* params, uint64_t d, uint64_t dim, const float* xp, uint64_t n,
                               int32_t device, float* out);
/* Gradient of the mean squared error of one batch (batch a multiple of 128): out_grads in the flat
 * parameter layout, out_loss the loss (the check against a CPU oracle). */
pacmap_status pacmap_mlp_grad(const float* params, uint64_t d, uint64_t dim, const float* xp, const float* target,
                              uint64_t batch, int32_t device, float* out_grads, float* out_loss);
/* fit_transform (src/lib.rs:294-367) with the learned initialiser; cfg->init_kind is ignored, pass a
 * shortened cfg->num_iters. target_mean, target_std (dim values each, host; see pacmap_model_target_stats):
 * the training embedding's per-dimension mean and std -- given, the fit starts from MLP(x') * std + mean,
 * the training embedding's coordinates (where pacmap_transform places new points), so the predicted
 * layout survives the first Adam steps; NULL (both), it starts from MLP(x') through Initialization::Value
 * (src/lib.rs:753-766: z-scored to std 1e-4 like any Value init). */
pacmap_status pacmap_fit_transform_learned(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                           const float* mlp_params, const float* target_mean, const float* target_std,
                                           float* out_embedding, float* out_snapshots);
pacmap_status pacmap_fit_transform_learned_device(const float* d_x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                                  const float* mlp_params, const float* target_mean,
                                                  const float* target_std, float* d_out_embedding,
                                                  float* d_out_snapshots);

/* Initialization::Pca's eigen-step on the host (no GPU): the k leading eigenvectors of a symmetric
 * d x d matrix (f64, row-major) into axes (d x k, row-major), by descending eigenvalue, each column's
 * largest-magnitude entry positive. Cyclic Jacobi for d <= 160, else subspace iteration + Rayleigh-Ritz. */
pacmap_status pacmap_pca_axes(const double* cov, uint64_t d, uint64_t k, double* out_axes);

/* --- the learned model on disk and the transform of new points (no reference analogue: the reference
 * embeds only the points it was fitted on, README.md:165) ---
 * A model is the MLP above, its training data's preprocessing constants (pacmap_preprocess's min, max
 * and column means) and the per-dimension mean and standard deviation of the training embedding (the
 * network predicts z-scored coordinates). */
/* out_mean, out_std (dim values each) of an embedding y (n x dim): the standardisation that
 * pacmap_mlp_train applies to its targets. */
pacmap_status pacmap_model_target_stats(const float* y, uint64_t n, uint64_t dim, float* out_mean, float* out_std);
/* Writes a model file (format in pacmap-rs_b200/csrc/model.cu; checksummed). params: the flat layout
 * of pacmap_mlp_param_count(d, dim) values; pre_mean: d values; target_mean, target_std: dim values. */
pacmap_status pacmap_model_save(const char* path, uint64_t d, uint64_t dim, const float* params, float pre_min,
                                float pre_max, const float* pre_mean, const float* target_mean,
                                const float* target_std);
/* Reads a model file; every output may be NULL (read out_d and out_dim first, then size the buffers).
 * A damaged, truncated or foreign file returns PACMAP_ERR_MODEL_FILE. */
pacmap_status pacmap_model_load(const char* path, uint64_t* out_d, uint64_t* out_dim, float* out_params,
                                float* out_pre_min, float* out_pre_max, float* out_pre_mean,
                                float* out_target_mean, float* out_target_std);
/* Embeds new points x (n x d, raw data like the training data) into the training embedding's
 * coordinates: x' = (x - pre_min) / pre_max - pre_mean (preprocess_x's f32 arithmetic with the stored
 * constants), then out (n x dim) = MLP(x') * target_std + target_mean. */
pacmap_status pacmap_transform(const float* x, uint64_t n, uint64_t d, uint64_t dim, const float* params,
                               float pre_min, float pre_max, const float* pre_mean, const float* target_mean,
                               const float* target_std, int32_t device, float* out_embedding);

/* Quality of an embedding (no reference analogue): mean 10-NN preservation over `sample` (n_sample
 * point indices; neighbours by the reference's f32 distance on the preprocessed data) and random-triplet
 * order accuracy over `triplets` (n_triplets x 3). x: raw n x d data; y: n x dim embedding. */
pacmap_status pacmap_quality(const float* x, uint64_t n, uint64_t d, const float* y, uint64_t dim,
                             const uint32_t* sample, uint64_t n_sample, uint64_t k, const uint32_t* triplets,
                             uint64_t n_triplets, int32_t device, double* out_preservation,
                             double* out_triplet_accuracy);

/* preprocess_x (the arithmetic of pacmap_preprocess) for callers that cannot allocate device memory --
 * a process whose device memory belongs to another framework's allocator or to a fixed budget, or a
 * latency-critical loop that must not reach cudaMalloc/cudaFree. No counterpart in the reference.
 * d_x, d_out: n x d device buffers on `device`; `stream` is a cudaStream_t (NULL = legacy default
 * stream). Stream-ordered: the call returns once the work is enqueued. The scratch is a fixed device
 * array of the library (at most 16,384 columns; larger d returns PACMAP_ERR_UNSUPPORTED), looked up on
 * the first call per device -- make that call before any stream capture -- and again on every call whose
 * stream is not capturing (the address belongs to the device's primary context). The caller's current
 * device is restored before the call returns. All calls share that array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
pacmap_status pacmap_preprocess_noalloc(const float* d_x, uint64_t n, uint64_t d, float* d_out, void* stream,
                                        int32_t device);

/* Stage timing (diagnostics): when enabled, each fit_transform records the device time of its stages
 * with CUDA events on its stream. pacmap_stage_times fills up to `cap` values in milliseconds, in the
 * order preprocess, knn, reselect, sample_mn, sample_fp, csr, init, optimize (then, when the tensor-core
 * kNN ran: its filter kernel alone, the number of rows it left to the exact fallback, the time of the
 * tile pruning's bound pass and lists, the (row block, column tile) pairs computed, of the full
 * sweep, and of the bound pass, and per row: candidate entries written by the filter passes, compactions
 * inside them, and candidates left for the exact re-rank; then the host milliseconds spent capturing and
 * instantiating the optimiser's CUDA graph, part of the optimize stage), and returns how many. */
void pacmap_set_stage_timing(int32_t enabled);
uint64_t pacmap_stage_times(double* out_ms, uint64_t cap);

/* The CUDA stream (cudaStream_t) on which every call for `device` enqueues its work, so that a caller
 * can time calls with events on the launching stream (no reference analogue); NULL on error. */
void* pacmap_device_stream(int32_t device);
/* The device's rate of random 8-byte loads from an L2-resident array, in loads per second (diagnostics,
 * no reference analogue): the ceiling of the gradient's partner gathers, one such load per CSR entry.
 * Runs for a few milliseconds. */
pacmap_status pacmap_gather_rate(int32_t device, double* out_loads_per_s);
/* Kernel launches issued by this thread since the last call of this function (diagnostics). */
uint64_t pacmap_take_launch_count(void);

/* Failure-detection test hook (no reference analogue; tests only). With on != 0, the tensor-core kNN
 * filter on `device` issues none of its operand copies, so its bounded wait on them runs out (2 s) and
 * every later kNN call fails with PACMAP_ERR_DEVICE_INVARIANT ("a bounded device wait timed out") instead
 * of hanging; on = 0 restores normal operation. The caller's current device is kept. */
pacmap_status pacmap_debug_stall_knn_loads(int32_t device, int32_t on);

/* The message of the last failure on this thread ("" after success). */
const char* pacmap_last_error(void);

/* Library version string. */
const char* pacmap_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PACMAP_B200_H */
