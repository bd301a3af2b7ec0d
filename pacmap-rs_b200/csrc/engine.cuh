// Host-side engine plumbing: per-call context, stream-ordered device buffers, stage launchers.
#pragma once

#include <vector>

#include "common.cuh"

namespace pacmap {

// One call's execution context: its device, its stream, and the device error word kernels OR into.
struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t* d_err = nullptr;  // device word (DevErr bits)
  int sm_count = 148;
  // Raise the bits of the device error word as a status (synchronises the stream).
  void check_errors(const char* stage);
};

// Stream-ordered device allocation (cudaMallocAsync on the call's stream; the device pool keeps freed
// blocks cached, so repeated calls do not pay for allocation). Every buffer starts on a 256-byte boundary,
// as cudaMalloc's do: the TMA tensor maps and the 16-byte vector loads rely on it.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t count = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(Ctx& c, size_t n) { alloc(c, n); }
  void alloc(Ctx& c, size_t n) {
    release();
    s = c.stream;
    count = n;
    if (n) PM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), n * sizeof(T), s));
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    count = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), count(o.count), s(o.s) { o.p = nullptr; o.count = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    p = o.p;
    count = o.count;
    s = o.s;
    o.p = nullptr;
    o.count = 0;
    return *this;
  }
  T* get() const { return p; }
  size_t bytes() const { return count * sizeof(T); }
};

// dst = a device copy of count host values (stream-ordered).
template <typename T>
void upload(Ctx& c, DevBuf<T>& dst, const T* src, size_t count) {
  dst.alloc(c, count);
  if (count) PM_CUDA(cudaMemcpyAsync(dst.get(), src, count * sizeof(T), cudaMemcpyHostToDevice, c.stream));
}

// ---- preprocess.cu ----
// preprocess_x non-PCA branch on the device; h_min/h_max receive the total-order extrema.
void preprocess_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float* d_out, float* h_min, float* h_max,
                       float* d_mean);
// mean_axis(Axis(0)) of ((x - sub) / div) in ndarray's sequential row order (sub = 0, div = 1 for plain x).
void column_mean_seq(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float sub, float div, float* d_mean);

// ---- knn.cu ----
// One shard of the query rows (multi-GPU kNN: every rank holds all points and computes its shard).
// The tensor-core path splits its row blocks (in the locality order), the SIMT path the rows in order;
// d_owned (n bytes, may be NULL) is set to 1 on the rows this shard wrote.
struct KnnShard {
  uint32_t index = 0, count = 1;
  uint8_t* d_owned = nullptr;
};
// Exact kNN (k' columns, ascending (f32 distance, index)) of the rows of d_x against all rows.
// mode PACMAP_KNN_APPROX searches approximately when n >= approx_threshold (exactly below it).
void knn_exact_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, int mode, uint32_t* d_idx,
                      float* d_dist, const KnnShard& shard = KnnShard(), uint64_t approx_threshold = 0);
// Exact kNN of a subset of rows (query ids in d_rows) against all rows.
// scatter: results go to the rows' own places (row r -> d_idx[r * kp]) instead of list order.
void knn_rows_simt(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, const uint32_t* d_rows,
                   uint64_t n_rows, uint32_t* d_idx, float* d_dist, bool scatter = false);

// ---- pairs.cu ----
void sigma_device(Ctx& c, const float* d_kd, uint64_t n, uint64_t kp, float* d_sig);
void reselect_device(Ctx& c, const uint32_t* d_nbr, const float* d_kd, const float* d_sig, uint64_t n, uint64_t kp,
                     uint64_t k, uint32_t* d_pnn);
void sample_mn_device(Ctx& c, const float* d_xp, uint64_t n, uint64_t d, uint64_t n_mn, uint64_t seed,
                      uint32_t* d_pmn);
void sample_fp_device(Ctx& c, const uint32_t* d_pnn, uint64_t n, uint64_t k, uint64_t n_fp, uint64_t seed,
                      uint32_t* d_pfp);

// ---- optimizer.cu ----
struct Csr {
  DevBuf<uint32_t> row_ptr;  // 3n + 1 offsets: segments (row, type) with type NN = 0, MN = 1, FP = 2
  DevBuf<uint32_t> col;      // partner of each entry, ascending within a segment
  uint64_t entries = 0;
};
// grouped_known: the lists are known to hold each point's pairs together (generated lists), so the
// device check of that (a kernel and a host round trip) is skipped.
void build_csr(Ctx& c, uint64_t n, const uint32_t* d_pnn, uint64_t n_nn, const uint32_t* d_pmn, uint64_t n_mn,
               const uint32_t* d_pfp, uint64_t n_fp, Csr& out, bool grouped_known = false);
void init_value_device(Ctx& c, const float* d_v, uint64_t n, uint64_t dim, float* d_y);

// Every row divided by its norm (the reference's f32 distance from the origin, distance.rs:50-75 order);
// zero rows stay zero. In place, n x d.
void normalize_rows_device(Ctx& c, float* d_x, uint64_t n, uint64_t d);

// ---- pca.cu: Initialization::Pca ----
// d_out (n x k) = scale * (x - column mean) V_k with V_k the k leading principal axes of x (n x d);
// axes_out (optional) receives V_k (d x k, row-major). k <= 128, d <= 1024.
void pca_project_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t k, float scale, float* d_out,
                        std::vector<float>* axes_out);
// The k leading eigenvectors of a symmetric d x d matrix (host, f64): axes (d x k, row-major), by
// descending eigenvalue, each column's largest-magnitude entry positive.
void pca_top_axes(const double* cov, uint64_t d, uint64_t k, double* axes);
// d_out (n x k) = scale * x[:, :k] for x (n x w).
void leading_columns(Ctx& c, const float* d_x, uint64_t n, uint64_t w, uint64_t k, float scale, float* d_out);
void init_random_device(Ctx& c, uint64_t n, uint64_t dim, uint64_t seed, float* d_y);

struct OptimizeArgs {
  float* d_y = nullptr;  // n x dim, in: state at itr_begin, out: state at itr_end
  float* d_m = nullptr;
  float* d_v = nullptr;
  uint64_t n = 0, dim = 0;
  float lr = 1.0f;
  uint64_t p1 = 100, p2 = 100, p3 = 250;
  uint64_t itr_begin = 0, itr_end = 450;
  const uint64_t* snapshots = nullptr;  // host list, may be NULL
  uint64_t n_snapshots = 0;
  float* d_snap = nullptr;              // n_snapshots x n x dim (slot 0 pre-filled by the caller)
  float* h_loss = nullptr;              // per-iteration loss (host, itr_end - itr_begin values), may be NULL
  float* d_grad_last = nullptr;         // (n+1) x dim gradient of the last iteration, may be NULL
};
void optimize_device(Ctx& c, const Csr& csr, const OptimizeArgs& a);
// Host milliseconds the last optimize_device on this thread spent capturing and instantiating its graph.
double& last_graph_setup_ms();
// One gradient evaluation with explicit weights: d_grad (n x dim), *h_loss the loss.
void gradient_device(Ctx& c, const Csr& csr, const float* d_y, uint64_t n, uint64_t dim, float w_nn, float w_mn,
                     float w_fp, float* d_grad, float* h_loss);

// ---- metrics.cu ----
// Random 8-byte loads per second from an L2-resident 8 MB array (best of 3 timed launches).
double gather_rate_device(Ctx& c);
void quality_device(Ctx& c, const float* d_xp, uint64_t n, uint64_t d, const float* d_y, uint64_t dim,
                    const uint32_t* d_sample, uint64_t n_sample, uint64_t k, const uint32_t* d_trip,
                    uint64_t n_trip, double* h_pres, double* h_trip);

}  // namespace pacmap
