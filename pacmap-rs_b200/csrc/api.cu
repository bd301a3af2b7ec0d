// C ABI of the engine (include/pacmap.h): validation in the reference's order, host<->device copies,
// and the stage sequence of fit_transform (src/lib.rs:294-367).
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "engine.cuh"
#include "knn_tc.cuh"
#include "mlp.cuh"

namespace pacmap {

namespace {
thread_local std::string g_last_error;
thread_local uint64_t g_launches = 0;
thread_local bool g_stage_timing = false;
thread_local std::vector<double> g_stage_ms;
std::mutex g_device_mutex[64];

struct DeviceState {
  bool ready = false;
  cudaStream_t stream = nullptr;
  uint32_t* d_err = nullptr;
  int sm_count = 148;
};
DeviceState g_devices[64];
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
void count_launch(uint64_t k) { g_launches += k; }

void Ctx::check_errors(const char* stage) {
  uint32_t h = 0;
  PM_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  PM_CUDA(cudaStreamSynchronize(stream));
  if (h == 0) return;
  PM_CUDA(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), stream));
  PM_CUDA(cudaStreamSynchronize(stream));
  const std::string where = std::string(" (") + stage + ")";
  if (h & DEV_ERR_PAIR_INDEX) throw Fail{PACMAP_ERR_PAIR_INDEX, "a pair index is out of range [0, n)" + where};
  if (h & DEV_ERR_SAMPLING)
    throw Fail{PACMAP_ERR_SAMPLING, "cannot draw the requested distinct partners (duplicated exclusions?)" + where};
  if (h & DEV_ERR_TIMEOUT) throw Fail{PACMAP_ERR_DEVICE_INVARIANT, "a bounded device wait timed out" + where};
  throw Fail{PACMAP_ERR_DEVICE_INVARIANT, "device invariant violated, code " + std::to_string(h) + where};
}

namespace {

// Locks the device for the duration of a call and hands out its stream and error word.
struct DeviceLock {
  std::unique_lock<std::mutex> lock;
  Ctx ctx;
  explicit DeviceLock(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Fail{PACMAP_ERR_NO_DEVICE, "no CUDA device is visible"};
    }
    if (device < 0 || device >= count || device >= 64)
      throw Fail{PACMAP_ERR_INVALID_ARGUMENT, "device ordinal " + std::to_string(device) + " is not available"};
    lock = std::unique_lock<std::mutex>(g_device_mutex[device]);
    PM_CUDA(cudaSetDevice(device));
    DeviceState& st = g_devices[device];
    if (!st.ready) {
      cudaDeviceProp prop;
      PM_CUDA(cudaGetDeviceProperties(&prop, device));
      if (prop.major != 10)
        throw Fail{PACMAP_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not compute capability 10.x (sm_100)"};
      PM_CUDA(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
      PM_CUDA(cudaMalloc(&st.d_err, sizeof(uint32_t)));
      PM_CUDA(cudaMemset(st.d_err, 0, sizeof(uint32_t)));
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      }
      st.sm_count = prop.multiProcessorCount;
      st.ready = true;
    }
    ctx.device = device;
    ctx.stream = st.stream;
    ctx.d_err = st.d_err;
    ctx.sm_count = st.sm_count;
  }
};

template <typename F>
pacmap_status guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return PACMAP_OK;
  } catch (const Fail& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return PACMAP_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return PACMAP_ERR_INVALID_ARGUMENT;
  }
}

// Rust `f as usize` (saturating, NaN -> 0).
uint64_t f32_as_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 18446744073709551616.0f) return UINT64_MAX;
  return static_cast<uint64_t>(f);
}

struct PairCounts {
  uint64_t k, n_mn, n_fp;
};

// src/lib.rs:565-597 decide_num_pairs in the reference's f32 arithmetic.
PairCounts decide_num_pairs(uint64_t n, const pacmap_config& cfg) {
  uint64_t k;
  if (cfg.has_override_neighbors) {
    k = cfg.override_neighbors;
  } else if (n <= 10000) {
    k = 10;
  } else {
    k = f32_as_usize(std::round(10.0f + 15.0f * (std::log10(static_cast<float>(n)) - 4.0f)));
  }
  const uint64_t n_mn = f32_as_usize(std::round(static_cast<float>(k) * cfg.mid_near_ratio));
  const uint64_t n_fp = f32_as_usize(std::round(static_cast<float>(k) * cfg.far_pair_ratio));
  PM_REQUIRE(k >= 1, PACMAP_ERR_INVALID_NEIGHBOR_COUNT, "The number of nearest neighbors can't be less than 1");
  PM_REQUIRE(n_fp >= 1, PACMAP_ERR_INVALID_FAR_POINT_COUNT, "The number of far points can't be less than 1");
  return {k, n_mn, n_fp};
}

uint64_t entropy_seed() {
  std::random_device rd;
  return (static_cast<uint64_t>(rd()) << 32) ^ rd();
}

// Device-time marks between the stages of one call (CUDA events on the call's stream).
enum Stage { ST_PRE = 0, ST_KNN, ST_RESELECT, ST_MN, ST_FP, ST_CSR, ST_INIT, ST_OPT, ST_COUNT };
struct StageTimer {
  cudaStream_t s = nullptr;
  cudaEvent_t ev[ST_COUNT + 1] = {};
  bool on = false;
  explicit StageTimer(cudaStream_t stream) : s(stream), on(g_stage_timing) {
    if (!on) return;
    for (auto& e : ev) PM_CUDA(cudaEventCreate(&e));
    g_stage_ms.assign(ST_COUNT, 0.0);  // + knn_filter ms and fallback rows appended by the kNN stage
  }
  void start(int stage) {
    if (on) PM_CUDA(cudaEventRecord(ev[stage], s));
  }
  void stop(int stage) {
    if (!on) return;
    PM_CUDA(cudaEventRecord(ev[ST_COUNT], s));
    PM_CUDA(cudaEventSynchronize(ev[ST_COUNT]));
    float ms = 0.0f;
    PM_CUDA(cudaEventElapsedTime(&ms, ev[stage], ev[ST_COUNT]));
    g_stage_ms[stage] += ms;
  }
  ~StageTimer() {
    if (on)
      for (auto& e : ev) cudaEventDestroy(e);
  }
};

struct DevPairs {
  DevBuf<uint32_t> nn, mn, fp;
  uint64_t n_nn = 0, n_mn = 0, n_fp = 0;  // rows
};

// neighbors.rs:56-108 generate_pairs on the preprocessed data (exact kNN at every n).
void generate_pairs_device(Ctx& c, const float* d_xp, uint64_t n, uint64_t d, const PairCounts& pc, uint64_t seed,
                           int knn_mode, DevPairs& out, StageTimer* tm = nullptr, uint64_t approx_threshold = 0) {
  const uint64_t kp = std::min<uint64_t>(pc.k + 50, n - 1);
  const uint64_t k = std::min<uint64_t>(pc.k, n - 1);
  DevBuf<uint32_t> idx(c, n * kp);
  DevBuf<float> dist(c, n * kp), sig(c, n);
  if (tm) tm->start(ST_KNN);
  last_tc_stats() = KnnTcStats();
  knn_exact_device(c, d_xp, n, d, kp, knn_mode, idx.get(), dist.get(), KnnShard(), approx_threshold);
  if (tm) tm->stop(ST_KNN);
  if (tm && tm->on) {
    const KnnTcStats& ks = last_tc_stats();
    g_stage_ms.resize(ST_COUNT + 9, 0.0);
    g_stage_ms[ST_COUNT] = ks.filter_ms;
    g_stage_ms[ST_COUNT + 1] = static_cast<double>(ks.fallback_rows);
    g_stage_ms[ST_COUNT + 2] = ks.bound_ms;
    g_stage_ms[ST_COUNT + 3] = static_cast<double>(ks.tiles_visited);
    g_stage_ms[ST_COUNT + 4] = static_cast<double>(ks.tiles_full);
    g_stage_ms[ST_COUNT + 5] = static_cast<double>(ks.tiles_bound);
    const double rows = ks.rows ? static_cast<double>(ks.rows) : 1.0;
    g_stage_ms[ST_COUNT + 6] = static_cast<double>(ks.insertions) / rows;
    g_stage_ms[ST_COUNT + 7] = static_cast<double>(ks.compactions) / rows;
    g_stage_ms[ST_COUNT + 8] = static_cast<double>(ks.band_entries) / rows;
  }
  if (tm) tm->start(ST_RESELECT);
  sigma_device(c, dist.get(), n, kp, sig.get());
  out.nn.alloc(c, n * k * 2);
  out.n_nn = n * k;
  reselect_device(c, idx.get(), dist.get(), sig.get(), n, kp, k, out.nn.get());
  if (tm) tm->stop(ST_RESELECT);
  out.mn.alloc(c, n * pc.n_mn * 2);
  out.n_mn = n * pc.n_mn;
  if (tm) tm->start(ST_MN);
  sample_mn_device(c, d_xp, n, d, pc.n_mn, seed, out.mn.get());
  if (tm) tm->stop(ST_MN);
  out.fp.alloc(c, n * pc.n_fp * 2);
  out.n_fp = n * pc.n_fp;
  if (tm) tm->start(ST_FP);
  sample_fp_device(c, out.nn.get(), n, k, pc.n_fp, seed, out.fp.get());
  if (tm) tm->stop(ST_FP);
  c.check_errors("pair sampling");
}

void validate_config(const pacmap_config* cfg) {
  PM_REQUIRE(cfg != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "config is NULL");
  PM_REQUIRE(cfg->init_kind >= 0 && cfg->init_kind <= 2, PACMAP_ERR_INVALID_ARGUMENT, "unknown init_kind");
  PM_REQUIRE(cfg->pair_kind >= 0 && cfg->pair_kind <= 2, PACMAP_ERR_INVALID_ARGUMENT, "unknown pair_kind");
  PM_REQUIRE(cfg->knn_mode >= 0 && cfg->knn_mode <= 5, PACMAP_ERR_INVALID_ARGUMENT, "unknown knn_mode");
  PM_REQUIRE(cfg->metric == PACMAP_METRIC_EUCLIDEAN || cfg->metric == PACMAP_METRIC_ANGULAR,
             PACMAP_ERR_INVALID_ARGUMENT, "unknown metric");
}

// preprocess_x (src/lib.rs:442-522): the normalised data, or -- with Initialization::Pca and more than 100
// columns (:455) -- the projection onto min(100, n) principal axes, on which the pairs are then drawn
// (pca_solution). Returns the working data's column count.
// With the angular metric the working rows are then scaled to unit norm.
uint64_t preprocess_for(Ctx& c, const float* d_x, uint64_t n, uint64_t d, const pacmap_config& cfg, bool learned,
                        DevBuf<float>& xp) {
  uint64_t w = d;
  if (cfg.init_kind == PACMAP_INIT_PCA && !learned && d > 100) {
    w = std::min<uint64_t>(100, n);
    xp.alloc(c, n * w);
    pca_project_device(c, d_x, n, d, w, 1.0f, xp.get(), nullptr);
  } else {
    xp.alloc(c, n * d);
    preprocess_device(c, d_x, n, d, xp.get(), nullptr, nullptr, nullptr);
  }
  if (cfg.metric == PACMAP_METRIC_ANGULAR) normalize_rows_device(c, xp.get(), n, w);
  return w;
}

// fit_transform with x already on the device; h_* pointers are the caller's host views of the config.
void fit_transform_impl(Ctx& c, const float* d_x, uint64_t n, uint64_t d, const pacmap_config& cfg, float* d_out,
                        float* d_snap, const float* mlp_params = nullptr, const float* t_mean = nullptr,
                        const float* t_std = nullptr) {
  // lib.rs:300-302
  PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
  const uint64_t dim = cfg.embedding_dimensions;
  PM_REQUIRE(dim <= 8, PACMAP_ERR_UNSUPPORTED, "embedding dimensions above 8 are not supported");
  StageTimer tm(c.stream);
  // lib.rs:442-522 (the PCA branch is never taken: init is Value or Random)
  DevBuf<float> xp;
  tm.start(ST_PRE);
  const uint64_t dw = preprocess_for(c, d_x, n, d, cfg, mlp_params != nullptr, xp);
  tm.stop(ST_PRE);
  // lib.rs:333-338
  const PairCounts pc = decide_num_pairs(n, cfg);
  const uint64_t seed = cfg.has_seed ? cfg.seed : entropy_seed();
  // lib.rs:629-692 sample_pairs
  DevPairs pairs;
  if (cfg.pair_kind == PACMAP_PAIRS_GENERATE) {
    generate_pairs_device(c, xp.get(), n, dw, pc, seed, cfg.knn_mode, pairs, &tm, cfg.approx_threshold);
  } else if (cfg.pair_kind == PACMAP_PAIRS_NEIGHBORS_PROVIDED) {
    const uint64_t expected = n * pc.k;
    if (cfg.pair_neighbors_rows != expected)
      throw Fail{PACMAP_ERR_INVALID_NN_SHAPE, "Invalid shape for nearest neighbor pairs. Expected [" +
                                                  std::to_string(expected) + ", 2], got [" +
                                                  std::to_string(cfg.pair_neighbors_rows) + ", 2]"};
    PM_REQUIRE(cfg.pair_neighbors != nullptr || expected == 0, PACMAP_ERR_INVALID_ARGUMENT, "pair_neighbors is NULL");
    upload(c, pairs.nn, cfg.pair_neighbors, expected * 2);
    pairs.n_nn = expected;
    pairs.mn.alloc(c, n * pc.n_mn * 2);
    pairs.n_mn = n * pc.n_mn;
    sample_mn_device(c, xp.get(), n, dw, pc.n_mn, seed, pairs.mn.get());
    pairs.fp.alloc(c, n * pc.n_fp * 2);
    pairs.n_fp = n * pc.n_fp;
    sample_fp_device(c, pairs.nn.get(), n, pc.k, pc.n_fp, seed, pairs.fp.get());
    c.check_errors("pair sampling");
  } else {
    PM_REQUIRE((cfg.pair_neighbors || !cfg.pair_neighbors_rows) && (cfg.pair_mn || !cfg.pair_mn_rows) &&
                   (cfg.pair_fp || !cfg.pair_fp_rows),
               PACMAP_ERR_INVALID_ARGUMENT, "a provided pair list is NULL");
    upload(c, pairs.nn, cfg.pair_neighbors, cfg.pair_neighbors_rows * 2);
    upload(c, pairs.mn, cfg.pair_mn, cfg.pair_mn_rows * 2);
    upload(c, pairs.fp, cfg.pair_fp, cfg.pair_fp_rows * 2);
    pairs.n_nn = cfg.pair_neighbors_rows;
    pairs.n_mn = cfg.pair_mn_rows;
    pairs.n_fp = cfg.pair_fp_rows;
  }
  if (dim == 0) return;
  // lib.rs:752-779 initial embedding
  tm.start(ST_INIT);
  if (mlp_params && t_mean && t_std) {
    // learned initialiser in the training embedding's coordinates: MLP(x') * std + mean, where the plain
    // schedule would have placed the points (the network predicts standardised coordinates)
    mlp_apply_device(c, mlp_params, d, dim, xp.get(), n, d_out);
    destandardise_device(c, d_out, n, dim, t_mean, t_std);
  } else if (mlp_params) {
    // learned initialiser: MLP(x') as Initialization::Value (lib.rs:753-766 z-scores it to std 1e-4)
    DevBuf<float> raw(c, n * dim);
    mlp_apply_device(c, mlp_params, d, dim, xp.get(), n, raw.get());
    init_value_device(c, raw.get(), n, dim, d_out);
  } else if (cfg.init_kind == PACMAP_INIT_PCA) {
    if (dw != d) {
      // YInit::Preprocessed (lib.rs:765): 0.01 * the leading columns of the PCA projection
      PM_REQUIRE(dim <= dw, PACMAP_ERR_PCA, "PCA: more embedding dimensions than principal components");
      leading_columns(c, xp.get(), n, dw, dim, 0.01f, d_out);
    } else {
      // YInit::DimensionalReduction (lib.rs:766): Pca(min(n, dim)) fitted on x', its transform * 0.01
      PM_REQUIRE(dim <= d && dim <= n, PACMAP_ERR_PCA,
                 "PCA: the embedding needs no more dimensions than the data has columns and rows");
      pca_project_device(c, xp.get(), n, d, dim, 0.01f, d_out, nullptr);
    }
  } else if (cfg.init_kind == PACMAP_INIT_VALUE) {
    PM_REQUIRE(cfg.init_value != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "init_value is NULL");
    DevBuf<float> v;
    upload(c, v, cfg.init_value, n * dim);
    init_value_device(c, v.get(), n, dim, d_out);
  } else {
    init_random_device(c, n, dim, cfg.init_has_seed ? cfg.init_seed : entropy_seed(), d_out);
  }
  if (d_snap && cfg.snapshots && cfg.n_snapshots > 0) {
    PM_CUDA(cudaMemsetAsync(d_snap, 0, cfg.n_snapshots * n * dim * sizeof(float), c.stream));
    PM_CUDA(cudaMemcpyAsync(d_snap, d_out, n * dim * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
  }
  tm.stop(ST_INIT);
  Csr csr;
  tm.start(ST_CSR);
  // generated lists come out grouped by point (no device check needed); provided ones are checked
  build_csr(c, n, pairs.nn.get(), pairs.n_nn, pairs.mn.get(), pairs.n_mn, pairs.fp.get(), pairs.n_fp, csr,
            cfg.pair_kind == PACMAP_PAIRS_GENERATE);
  tm.stop(ST_CSR);
  DevBuf<float> m(c, n * dim), v(c, n * dim);
  PM_CUDA(cudaMemsetAsync(m.get(), 0, n * dim * sizeof(float), c.stream));
  PM_CUDA(cudaMemsetAsync(v.get(), 0, n * dim * sizeof(float), c.stream));
  OptimizeArgs a;
  a.d_y = d_out;
  a.d_m = m.get();
  a.d_v = v.get();
  a.n = n;
  a.dim = dim;
  a.lr = cfg.learning_rate;
  a.p1 = cfg.num_iters[0];
  a.p2 = cfg.num_iters[1];
  a.p3 = cfg.num_iters[2];
  a.itr_begin = 0;
  a.itr_end = a.p1 + a.p2 + a.p3;
  a.snapshots = cfg.snapshots;
  a.n_snapshots = cfg.n_snapshots;
  a.d_snap = d_snap;
  a.h_loss = cfg.loss_trace;
  tm.start(ST_OPT);
  optimize_device(c, csr, a);
  tm.stop(ST_OPT);
  if (tm.on) {
    g_stage_ms.resize(std::max<size_t>(g_stage_ms.size(), ST_COUNT + 10), 0.0);
    g_stage_ms[ST_COUNT + 9] = last_graph_setup_ms();
  }
  c.check_errors("optimiser");
}

}  // namespace
}  // namespace pacmap

using namespace pacmap;

extern "C" {

const char* pacmap_last_error(void) { return g_last_error.c_str(); }
const char* pacmap_version(void) { return "pacmap-b200 0.1.0 (sm_100a)"; }

void pacmap_set_stage_timing(int32_t enabled) { g_stage_timing = enabled != 0; }

uint64_t pacmap_stage_times(double* out_ms, uint64_t cap) {
  const uint64_t k = std::min<uint64_t>(cap, g_stage_ms.size());
  for (uint64_t i = 0; i < k; ++i) out_ms[i] = g_stage_ms[i];
  return g_stage_ms.size();
}

void* pacmap_device_stream(int32_t device) {
  try {
    DeviceLock dl(device);
    return static_cast<void*>(dl.ctx.stream);
  } catch (const Fail& f) {
    set_last_error(f.msg);
    return nullptr;
  }
}

uint64_t pacmap_take_launch_count(void) {
  const uint64_t v = g_launches;
  g_launches = 0;
  return v;
}

pacmap_config pacmap_config_default(void) {
  pacmap_config c;
  std::memset(&c, 0, sizeof(c));
  c.embedding_dimensions = 2;
  c.init_kind = PACMAP_INIT_PCA;
  c.mid_near_ratio = 0.5f;
  c.far_pair_ratio = 2.0f;
  c.pair_kind = PACMAP_PAIRS_GENERATE;
  c.learning_rate = 1.0f;
  c.num_iters[0] = 100;
  c.num_iters[1] = 100;
  c.num_iters[2] = 250;
  c.approx_threshold = 8000;
  c.knn_mode = PACMAP_KNN_AUTO;
  c.device = 0;
  c.metric = PACMAP_METRIC_EUCLIDEAN;
  return c;
}

pacmap_status pacmap_fit_transform(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                   float* out_embedding, float* out_snapshots) {
  return guarded([&] {
    validate_config(cfg);
    PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
    PM_REQUIRE(x != nullptr && (out_embedding != nullptr || cfg->embedding_dimensions == 0),
               PACMAP_ERR_INVALID_ARGUMENT, "x or out_embedding is NULL");
    DeviceLock dl(cfg->device);
    Ctx& c = dl.ctx;
    const uint64_t dim = cfg->embedding_dimensions;
    DevBuf<float> dx, dy(c, n * dim), ds;
    upload(c, dx, x, n * d);
    const bool snaps = out_snapshots && cfg->snapshots && cfg->n_snapshots > 0;
    if (snaps) ds.alloc(c, cfg->n_snapshots * n * dim);
    fit_transform_impl(c, dx.get(), n, d, *cfg, dy.get(), snaps ? ds.get() : nullptr);
    if (dim) PM_CUDA(cudaMemcpyAsync(out_embedding, dy.get(), n * dim * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    if (snaps)
      PM_CUDA(cudaMemcpyAsync(out_snapshots, ds.get(), ds.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_fit_transform_device(const float* d_x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                          float* d_out_embedding, float* d_out_snapshots) {
  return guarded([&] {
    validate_config(cfg);
    PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
    PM_REQUIRE(d_x != nullptr && (d_out_embedding != nullptr || cfg->embedding_dimensions == 0),
               PACMAP_ERR_INVALID_ARGUMENT, "x or out_embedding is NULL");
    DeviceLock dl(cfg->device);
    fit_transform_impl(dl.ctx, d_x, n, d, *cfg, d_out_embedding, d_out_snapshots);
    PM_CUDA(cudaStreamSynchronize(dl.ctx.stream));
  });
}

pacmap_status pacmap_fit_transform_learned(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                           const float* mlp_params, const float* target_mean, const float* target_std,
                                           float* out_embedding, float* out_snapshots) {
  return guarded([&] {
    validate_config(cfg);
    PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
    PM_REQUIRE(x && mlp_params && out_embedding, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(cfg->device);
    Ctx& c = dl.ctx;
    const uint64_t dim = cfg->embedding_dimensions;
    DevBuf<float> dx, dy(c, n * dim), ds;
    upload(c, dx, x, n * d);
    const bool snaps = out_snapshots && cfg->snapshots && cfg->n_snapshots > 0;
    if (snaps) ds.alloc(c, cfg->n_snapshots * n * dim);
    PM_REQUIRE((target_mean == nullptr) == (target_std == nullptr), PACMAP_ERR_INVALID_ARGUMENT,
               "target_mean and target_std go together");
    fit_transform_impl(c, dx.get(), n, d, *cfg, dy.get(), snaps ? ds.get() : nullptr, mlp_params, target_mean,
                       target_std);
    PM_CUDA(cudaMemcpyAsync(out_embedding, dy.get(), n * dim * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    if (snaps) PM_CUDA(cudaMemcpyAsync(out_snapshots, ds.get(), ds.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_fit_transform_learned_device(const float* d_x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                                  const float* mlp_params, const float* target_mean,
                                                  const float* target_std, float* d_out_embedding,
                                                  float* d_out_snapshots) {
  return guarded([&] {
    validate_config(cfg);
    PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
    PM_REQUIRE(d_x && mlp_params && d_out_embedding, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(cfg->device);
    PM_REQUIRE((target_mean == nullptr) == (target_std == nullptr), PACMAP_ERR_INVALID_ARGUMENT,
               "target_mean and target_std go together");
    fit_transform_impl(dl.ctx, d_x, n, d, *cfg, d_out_embedding, d_out_snapshots, mlp_params, target_mean,
                       target_std);
    PM_CUDA(cudaStreamSynchronize(dl.ctx.stream));
  });
}

uint64_t pacmap_mlp_param_count(uint64_t d, uint64_t dim) { return mlp_param_count(d, dim); }

pacmap_status pacmap_mlp_init(uint64_t d, uint64_t dim, uint64_t seed, float* out_params) {
  return guarded([&] {
    PM_REQUIRE(out_params != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    mlp_init_params(d, dim, seed, out_params);
  });
}

pacmap_status pacmap_mlp_train(const float* xp, const float* target, uint64_t n, uint64_t d, uint64_t dim,
                               uint64_t epochs, uint64_t batch, float lr, float weight_decay, uint64_t seed,
                               int32_t device, float* inout_params, float* out_epoch_loss) {
  return guarded([&] {
    PM_REQUIRE(xp && target && inout_params, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(dim >= 1 && dim <= 16 && d >= 1 && d <= 4096, PACMAP_ERR_UNSUPPORTED, "MLP supports d <= 4096, dim <= 16");
    // targets z-scored per dimension: Initialization::Value rescales the output anyway (lib.rs:753-766)
    std::vector<float> t(target, target + n * dim);
    for (uint64_t cc = 0; cc < dim; ++cc) {
      double s = 0.0, s2 = 0.0;
      for (uint64_t i = 0; i < n; ++i) s += t[i * dim + cc];
      const double mu = s / static_cast<double>(n);
      for (uint64_t i = 0; i < n; ++i) s2 += (t[i * dim + cc] - mu) * (t[i * dim + cc] - mu);
      const double sd = std::sqrt(s2 / static_cast<double>(n)) + 1e-30;
      for (uint64_t i = 0; i < n; ++i) t[i * dim + cc] = static_cast<float>((t[i * dim + cc] - mu) / sd);
    }
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dt;
    upload(c, dx, xp, n * d);
    upload(c, dt, t.data(), n * dim);
    mlp_train_device(c, inout_params, d, dim, dx.get(), dt.get(), n, epochs, batch, lr, weight_decay, seed,
                     out_epoch_loss);
  });
}

pacmap_status pacmap_mlp_apply(const float* params, uint64_t d, uint64_t dim, const float* xp, uint64_t n,
                               int32_t device, float* out) {
  return guarded([&] {
    PM_REQUIRE(params && xp && out, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dy(c, n * dim);
    upload(c, dx, xp, n * d);
    mlp_apply_device(c, params, d, dim, dx.get(), n, dy.get());
    PM_CUDA(cudaMemcpyAsync(out, dy.get(), dy.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_pca_axes(const double* cov, uint64_t d, uint64_t k, double* out_axes) {
  return guarded([&] {
    PM_REQUIRE(cov && out_axes, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    pca_top_axes(cov, d, k, out_axes);
  });
}

pacmap_status pacmap_model_target_stats(const float* y, uint64_t n, uint64_t dim, float* out_mean, float* out_std) {
  return guarded([&] {
    PM_REQUIRE(y && out_mean && out_std, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(n > 0, PACMAP_ERR_EMPTY_ARRAY_MEAN, "Failed to calculate mean axis: the array is empty");
    model_target_stats(y, n, dim, out_mean, out_std);
  });
}

pacmap_status pacmap_model_save(const char* path, uint64_t d, uint64_t dim, const float* params, float pre_min,
                                float pre_max, const float* pre_mean, const float* target_mean,
                                const float* target_std) {
  return guarded([&] {
    PM_REQUIRE(path && params && pre_mean && target_mean && target_std, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    model_save(path, d, dim, params, pre_min, pre_max, pre_mean, target_mean, target_std);
  });
}

pacmap_status pacmap_model_load(const char* path, uint64_t* out_d, uint64_t* out_dim, float* out_params,
                                float* out_pre_min, float* out_pre_max, float* out_pre_mean,
                                float* out_target_mean, float* out_target_std) {
  return guarded([&] {
    PM_REQUIRE(path != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "NULL path");
    model_load(path, out_d, out_dim, out_params, out_pre_min, out_pre_max, out_pre_mean, out_target_mean,
               out_target_std);
  });
}

pacmap_status pacmap_transform(const float* x, uint64_t n, uint64_t d, uint64_t dim, const float* params,
                               float pre_min, float pre_max, const float* pre_mean, const float* target_mean,
                               const float* target_std, int32_t device, float* out_embedding) {
  return guarded([&] {
    PM_REQUIRE(params && pre_mean && target_mean && target_std && (n == 0 || (x && out_embedding)),
               PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (n == 0) return;
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dy(c, n * dim);
    upload(c, dx, x, n * d);
    transform_device(c, dx.get(), n, d, dim, params, pre_min, pre_max, pre_mean, target_mean, target_std, dy.get());
    PM_CUDA(cudaMemcpyAsync(out_embedding, dy.get(), dy.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_mlp_grad(const float* params, uint64_t d, uint64_t dim, const float* xp, const float* target,
                              uint64_t batch, int32_t device, float* out_grads, float* out_loss) {
  return guarded([&] {
    PM_REQUIRE(params && xp && target && out_grads && out_loss, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dt;
    upload(c, dx, xp, batch * d);
    upload(c, dt, target, batch * dim);
    mlp_grad_device(c, params, d, dim, dx.get(), dt.get(), batch, out_grads, out_loss);
  });
}

pacmap_status pacmap_knn_exact(const float* x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode, int32_t device,
                               uint32_t* out_idx, float* out_dist) {
  return guarded([&] {
    if (n == 0) return;  // knn.rs:141-143
    const uint64_t kp = std::min<uint64_t>(k, n - 1);
    if (kp == 0) return;
    PM_REQUIRE(x && out_idx && out_dist, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(knn_mode >= 0 && knn_mode <= 5, PACMAP_ERR_INVALID_ARGUMENT, "unknown knn_mode");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dd(c, n * kp);
    DevBuf<uint32_t> di(c, n * kp);
    upload(c, dx, x, n * d);
    knn_exact_device(c, dx.get(), n, d, kp, knn_mode, di.get(), dd.get());
    PM_CUDA(cudaMemcpyAsync(out_idx, di.get(), di.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(out_dist, dd.get(), dd.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    c.check_errors("knn");
  });
}

pacmap_status pacmap_knn_exact_shard(const float* x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode,
                                     uint32_t shard, uint32_t n_shards, int32_t device, uint32_t* out_idx,
                                     float* out_dist, uint8_t* out_owned) {
  return guarded([&] {
    PM_REQUIRE(n_shards >= 1 && shard < n_shards, PACMAP_ERR_INVALID_ARGUMENT, "shard must be < n_shards");
    if (n == 0) return;
    const uint64_t kp = std::min<uint64_t>(k, n - 1);
    PM_REQUIRE(x && out_owned && (kp == 0 || (out_idx && out_dist)), PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(knn_mode >= 0 && knn_mode <= 5, PACMAP_ERR_INVALID_ARGUMENT, "unknown knn_mode");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dd(c, n * kp);
    DevBuf<uint32_t> di(c, n * kp);
    DevBuf<uint8_t> own(c, n);
    upload(c, dx, x, n * d);
    PM_CUDA(cudaMemsetAsync(own.get(), 0, n, c.stream));
    if (kp > 0) {
      PM_CUDA(cudaMemsetAsync(di.get(), 0, di.bytes(), c.stream));
      PM_CUDA(cudaMemsetAsync(dd.get(), 0, dd.bytes(), c.stream));
      KnnShard sh;
      sh.index = shard;
      sh.count = n_shards;
      sh.d_owned = own.get();
      knn_exact_device(c, dx.get(), n, d, kp, knn_mode, di.get(), dd.get(), sh);
      PM_CUDA(cudaMemcpyAsync(out_idx, di.get(), di.bytes(), cudaMemcpyDeviceToHost, c.stream));
      PM_CUDA(cudaMemcpyAsync(out_dist, dd.get(), dd.bytes(), cudaMemcpyDeviceToHost, c.stream));
    }
    PM_CUDA(cudaMemcpyAsync(out_owned, own.get(), n, cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    c.check_errors("knn shard");
  });
}

pacmap_status pacmap_knn_exact_shard_device(const float* d_x, uint64_t n, uint64_t d, uint64_t k, int32_t knn_mode,
                                            uint32_t shard, uint32_t n_shards, int32_t device, uint32_t* d_out_idx,
                                            float* d_out_dist, uint8_t* d_out_owned) {
  return guarded([&] {
    PM_REQUIRE(n_shards >= 1 && shard < n_shards, PACMAP_ERR_INVALID_ARGUMENT, "shard must be < n_shards");
    if (n == 0) return;
    const uint64_t kp = std::min<uint64_t>(k, n - 1);
    PM_REQUIRE(d_x && d_out_owned && (kp == 0 || (d_out_idx && d_out_dist)), PACMAP_ERR_INVALID_ARGUMENT,
               "NULL buffer");
    PM_REQUIRE(knn_mode >= 0 && knn_mode <= 5, PACMAP_ERR_INVALID_ARGUMENT, "unknown knn_mode");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    PM_CUDA(cudaMemsetAsync(d_out_owned, 0, n, c.stream));
    if (kp > 0) {
      PM_CUDA(cudaMemsetAsync(d_out_idx, 0, n * kp * sizeof(uint32_t), c.stream));
      PM_CUDA(cudaMemsetAsync(d_out_dist, 0, n * kp * sizeof(float), c.stream));
      KnnShard sh;
      sh.index = shard;
      sh.count = n_shards;
      sh.d_owned = d_out_owned;
      knn_exact_device(c, d_x, n, d, kp, knn_mode, d_out_idx, d_out_dist, sh);
    }
    PM_CUDA(cudaStreamSynchronize(c.stream));
    c.check_errors("knn shard");
  });
}

pacmap_status pacmap_preprocess(const float* x, uint64_t n, uint64_t d, int32_t device, float* out, float* out_min,
                                float* out_max, float* out_mean) {
  return guarded([&] {
    PM_REQUIRE(x && out, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, dout(c, n * d), dmean(c, d);
    upload(c, dx, x, n * d);
    preprocess_device(c, dx.get(), n, d, dout.get(), out_min, out_max, dmean.get());
    PM_CUDA(cudaMemcpyAsync(out, dout.get(), dout.bytes(), cudaMemcpyDeviceToHost, c.stream));
    if (out_mean) PM_CUDA(cudaMemcpyAsync(out_mean, dmean.get(), dmean.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_generate_pairs(const float* x, uint64_t n, uint64_t d, const pacmap_config* cfg,
                                    uint64_t* out_counts, uint32_t* out_pnn, uint32_t* out_pmn, uint32_t* out_pfp) {
  return guarded([&] {
    validate_config(cfg);
    PM_REQUIRE(n > 1, PACMAP_ERR_SAMPLE_SIZE, "Sample size must be larger than one");
    PM_REQUIRE(x != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "x is NULL");
    const PairCounts pc = decide_num_pairs(n, *cfg);
    if (out_counts) {
      out_counts[0] = std::min<uint64_t>(pc.k, n - 1);
      out_counts[1] = pc.n_mn;
      out_counts[2] = pc.n_fp;
    }
    if (!out_pnn && !out_pmn && !out_pfp) return;
    DeviceLock dl(cfg->device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, xp;
    upload(c, dx, x, n * d);
    const uint64_t dw = preprocess_for(c, dx.get(), n, d, *cfg, false, xp);
    DevPairs pairs;
    generate_pairs_device(c, xp.get(), n, dw, pc, cfg->has_seed ? cfg->seed : entropy_seed(), cfg->knn_mode, pairs,
                          nullptr, cfg->approx_threshold);
    if (out_pnn) PM_CUDA(cudaMemcpyAsync(out_pnn, pairs.nn.get(), pairs.nn.bytes(), cudaMemcpyDeviceToHost, c.stream));
    if (out_pmn) PM_CUDA(cudaMemcpyAsync(out_pmn, pairs.mn.get(), pairs.mn.bytes(), cudaMemcpyDeviceToHost, c.stream));
    if (out_pfp) PM_CUDA(cudaMemcpyAsync(out_pfp, pairs.fp.get(), pairs.fp.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_reselect_neighbors(const uint32_t* knn_idx, const float* knn_dist, uint64_t n, uint64_t kp,
                                        uint64_t k, int32_t device, uint32_t* out_pnn, float* out_sigma) {
  return guarded([&] {
    PM_REQUIRE(knn_idx && knn_dist && out_pnn, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(k <= kp, PACMAP_ERR_INVALID_ARGUMENT, "k must not exceed kp");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<uint32_t> di, dp(c, n * k * 2);
    DevBuf<float> dd, ds(c, n);
    upload(c, di, knn_idx, n * kp);
    upload(c, dd, knn_dist, n * kp);
    sigma_device(c, dd.get(), n, kp, ds.get());
    reselect_device(c, di.get(), dd.get(), ds.get(), n, kp, k, dp.get());
    PM_CUDA(cudaMemcpyAsync(out_pnn, dp.get(), dp.bytes(), cudaMemcpyDeviceToHost, c.stream));
    if (out_sigma) PM_CUDA(cudaMemcpyAsync(out_sigma, ds.get(), ds.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_sample_pairs(const float* xp, uint64_t n, uint64_t d, const uint32_t* pair_neighbors, uint64_t k,
                                  uint64_t n_mn, uint64_t n_fp, uint64_t seed, int32_t device, uint32_t* out_pmn,
                                  uint32_t* out_pfp) {
  return guarded([&] {
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    if (out_pmn && n_mn) {
      PM_REQUIRE(xp != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "xp is NULL");
      DevBuf<float> dx;
      DevBuf<uint32_t> dm(c, n * n_mn * 2);
      upload(c, dx, xp, n * d);
      sample_mn_device(c, dx.get(), n, d, n_mn, seed, dm.get());
      PM_CUDA(cudaMemcpyAsync(out_pmn, dm.get(), dm.bytes(), cudaMemcpyDeviceToHost, c.stream));
      PM_CUDA(cudaStreamSynchronize(c.stream));
    }
    if (out_pfp && n_fp) {
      PM_REQUIRE(pair_neighbors != nullptr || k == 0, PACMAP_ERR_INVALID_ARGUMENT, "pair_neighbors is NULL");
      DevBuf<uint32_t> dn, df(c, n * n_fp * 2);
      upload(c, dn, pair_neighbors, n * k * 2);
      sample_fp_device(c, dn.get(), n, k, n_fp, seed, df.get());
      PM_CUDA(cudaMemcpyAsync(out_pfp, df.get(), df.bytes(), cudaMemcpyDeviceToHost, c.stream));
      PM_CUDA(cudaStreamSynchronize(c.stream));
    }
    c.check_errors("pair sampling");
  });
}

pacmap_status pacmap_optimize_steps(float* y, float* m, float* v, uint64_t n, uint64_t dim, const uint32_t* pnn,
                                    uint64_t n_nn, const uint32_t* pmn, uint64_t n_mn, const uint32_t* pfp,
                                    uint64_t n_fp, float learning_rate, uint64_t p1, uint64_t p2, uint64_t itr_begin,
                                    uint64_t itr_end, int32_t device, float* out_grad) {
  return guarded([&] {
    PM_REQUIRE(y && m && v, PACMAP_ERR_INVALID_ARGUMENT, "NULL state buffer");
    PM_REQUIRE(dim >= 1 && dim <= 8, PACMAP_ERR_UNSUPPORTED, "the optimiser supports embedding dimensions 1..8");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dy, dm, dv, dg;
    DevBuf<uint32_t> a, b, e;
    upload(c, dy, y, n * dim);
    upload(c, dm, m, n * dim);
    upload(c, dv, v, n * dim);
    upload(c, a, pnn, n_nn * 2);
    upload(c, b, pmn, n_mn * 2);
    upload(c, e, pfp, n_fp * 2);
    Csr csr;
    build_csr(c, n, a.get(), n_nn, b.get(), n_mn, e.get(), n_fp, csr);
    std::vector<float> loss;
    OptimizeArgs oa;
    oa.d_y = dy.get();
    oa.d_m = dm.get();
    oa.d_v = dv.get();
    oa.n = n;
    oa.dim = dim;
    oa.lr = learning_rate;
    oa.p1 = p1;
    oa.p2 = p2;
    oa.p3 = 0;
    oa.itr_begin = itr_begin;
    oa.itr_end = itr_end;
    if (out_grad && itr_end > itr_begin) {
      dg.alloc(c, n * dim);
      oa.d_grad_last = dg.get();
      loss.resize(itr_end - itr_begin);
      oa.h_loss = loss.data();
    }
    optimize_device(c, csr, oa);
    c.check_errors("optimiser");
    PM_CUDA(cudaMemcpyAsync(y, dy.get(), dy.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(m, dm.get(), dm.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(v, dv.get(), dv.bytes(), cudaMemcpyDeviceToHost, c.stream));
    if (oa.d_grad_last)
      PM_CUDA(cudaMemcpyAsync(out_grad, dg.get(), dg.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    if (oa.d_grad_last) {
      out_grad[n * dim] = loss.back();
      for (uint64_t cc = 1; cc < dim; ++cc) out_grad[n * dim + cc] = 0.0f;
    }
  });
}

pacmap_status pacmap_gradient(const float* y, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn,
                              const uint32_t* pmn, uint64_t n_mn, const uint32_t* pfp, uint64_t n_fp, float w_nn,
                              float w_mn, float w_fp, int32_t device, float* out_grad) {
  return guarded([&] {
    PM_REQUIRE(y && out_grad, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(dim >= 1 && dim <= 8, PACMAP_ERR_UNSUPPORTED, "the optimiser supports embedding dimensions 1..8");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dy, dg(c, n * dim);
    DevBuf<uint32_t> a, b, e;
    upload(c, dy, y, n * dim);
    upload(c, a, pnn, n_nn * 2);
    upload(c, b, pmn, n_mn * 2);
    upload(c, e, pfp, n_fp * 2);
    Csr csr;
    build_csr(c, n, a.get(), n_nn, b.get(), n_mn, e.get(), n_fp, csr);
    float loss = 0.0f;
    gradient_device(c, csr, dy.get(), n, dim, w_nn, w_mn, w_fp, dg.get(), &loss);
    PM_CUDA(cudaMemcpyAsync(out_grad, dg.get(), dg.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    out_grad[n * dim] = loss;
    for (uint64_t cc = 1; cc < dim; ++cc) out_grad[n * dim + cc] = 0.0f;
  });
}

pacmap_status pacmap_init_value(const float* v, uint64_t n, uint64_t dim, int32_t device, float* out) {
  return guarded([&] {
    PM_REQUIRE(v && out, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dv, dy(c, n * dim);
    upload(c, dv, v, n * dim);
    init_value_device(c, dv.get(), n, dim, dy.get());
    PM_CUDA(cudaMemcpyAsync(out, dy.get(), dy.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_init_random(uint64_t n, uint64_t dim, uint64_t seed, int32_t device, float* out) {
  return guarded([&] {
    PM_REQUIRE(out, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dy(c, n * dim);
    init_random_device(c, n, dim, seed, dy.get());
    PM_CUDA(cudaMemcpyAsync(out, dy.get(), dy.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
  });
}

pacmap_status pacmap_gather_rate(int32_t device, double* out_loads_per_s) {
  return guarded([&] {
    PM_REQUIRE(out_loads_per_s, PACMAP_ERR_INVALID_ARGUMENT, "NULL output");
    DeviceLock dl(device);
    *out_loads_per_s = gather_rate_device(dl.ctx);
    dl.ctx.check_errors("gather rate");
  });
}

pacmap_status pacmap_quality(const float* x, uint64_t n, uint64_t d, const float* y, uint64_t dim,
                             const uint32_t* sample, uint64_t n_sample, uint64_t k, const uint32_t* triplets,
                             uint64_t n_triplets, int32_t device, double* out_preservation,
                             double* out_triplet_accuracy) {
  return guarded([&] {
    PM_REQUIRE(x && y, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE((sample || !n_sample) && (triplets || !n_triplets), PACMAP_ERR_INVALID_ARGUMENT, "NULL index list");
    for (uint64_t i = 0; i < n_sample; ++i)
      PM_REQUIRE(sample[i] < n, PACMAP_ERR_INVALID_ARGUMENT, "sample index out of range");
    for (uint64_t i = 0; i < 3 * n_triplets; ++i)
      PM_REQUIRE(triplets[i] < n, PACMAP_ERR_INVALID_ARGUMENT, "triplet index out of range");
    DeviceLock dl(device);
    Ctx& c = dl.ctx;
    DevBuf<float> dx, xp(c, n * d), dy;
    DevBuf<uint32_t> ds, dt;
    upload(c, dx, x, n * d);
    upload(c, dy, y, n * dim);
    upload(c, ds, sample, n_sample);
    upload(c, dt, triplets, n_triplets * 3);
    preprocess_device(c, dx.get(), n, d, xp.get(), nullptr, nullptr, nullptr);
    dx.release();
    quality_device(c, xp.get(), n, d, dy.get(), dim, ds.get(), n_sample, k, dt.get(), n_triplets, out_preservation,
                   out_triplet_accuracy);
  });
}

}  // extern "C"
