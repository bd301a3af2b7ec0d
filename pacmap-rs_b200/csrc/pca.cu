// Initialization::Pca (src/lib.rs:442-522, 753-768): principal axes of the data on the GPU.
//
// The reference calls petal-decomposition 0.8 (an exact SVD through LAPACK when d <= 100, a seeded
// randomized SVD otherwise); neither is in the reference tree. This file computes the exact principal
// axes -- the limit the randomized method approximates -- as eigenvectors of the covariance matrix:
//
//   1. column means (f64, fixed-order two-level sums);
//   2. the d x d covariance of the centred rows in f64: at most 64 row chunks (of at least 16,384 rows)
//      write 32 x 32 partial tiles, reduced over the chunks in order (deterministic, no atomics);
//   3. the top-k axes on the host (f64): cyclic Jacobi of the whole matrix for d <= 160, above that
//      subspace iteration on k + 24 vectors with a Rayleigh-Ritz step (the power iteration the
//      reference's randomized SVD uses); axes by descending variance, each axis's largest-magnitude
//      loading made positive (the reference's SVD sign is LAPACK's and unpinned);
//   4. the projection (x - mean) V_k by a tiled f32 kernel with f64 accumulation.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "engine.cuh"

namespace pacmap {
namespace {

constexpr int PCA_T = 32;           // covariance tile (32 x 32 outputs)
constexpr uint64_t PCA_MAX_CHUNKS = 64;  // partial covariances (row chunks of at least 16,384 rows)
constexpr int MEAN_BLOCKS = 256;

__global__ void __launch_bounds__(256) col_sum_partial_kernel(const float* __restrict__ x, uint64_t n, uint64_t d,
                                                              double* __restrict__ partial) {
  // block b sums rows [b * rpb, ...) of every column, each thread a strided set of columns
  const uint64_t rpb = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * rpb, r1 = r0 + rpb < n ? r0 + rpb : n;
  for (uint64_t c = threadIdx.x; c < d; c += blockDim.x) {
    double s = 0.0;
    for (uint64_t r = r0; r < r1; ++r) s += x[r * d + c];
    partial[static_cast<uint64_t>(blockIdx.x) * d + c] = s;
  }
}

__global__ void col_mean_final_kernel(const double* __restrict__ partial, int parts, uint64_t n, uint64_t d,
                                      double* __restrict__ mean) {
  const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= d) return;
  double s = 0.0;
  for (int b = 0; b < parts; ++b) s += partial[static_cast<uint64_t>(b) * d + c];
  mean[c] = s / static_cast<double>(n);
}

// Partial covariance of one row chunk for one 32 x 32 tile (ti, tj): thread (ty, tx) of a 32 x 8 block
// owns outputs (ti * 32 + ty, tj * 32 + tx + 8q), q < 4.
__global__ void __launch_bounds__(256) cov_partial_kernel(const float* __restrict__ x, uint64_t n, uint64_t d,
                                                          uint64_t rows_per_chunk, const double* __restrict__ mean,
                                                          double* __restrict__ partial) {
  __shared__ double a[PCA_T][PCA_T + 1], b[PCA_T][PCA_T + 1];  // [row][column]
  const int ti = blockIdx.x, tj = blockIdx.y;
  const uint64_t chunk = blockIdx.z;
  const uint64_t r0 = chunk * rows_per_chunk, r1 = r0 + rows_per_chunk < n ? r0 + rows_per_chunk : n;
  const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;  // ty 0..31
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint64_t rb = r0; rb < r1; rb += PCA_T) {
    __syncthreads();
    for (int e = threadIdx.x; e < PCA_T * PCA_T; e += 256) {
      const int rr = e / PCA_T, cc = e % PCA_T;
      const uint64_t r = rb + rr;
      const uint64_t ci = static_cast<uint64_t>(ti) * PCA_T + cc, cj = static_cast<uint64_t>(tj) * PCA_T + cc;
      a[rr][cc] = (r < r1 && ci < d) ? static_cast<double>(x[r * d + ci]) - mean[ci] : 0.0;
      b[rr][cc] = (r < r1 && cj < d) ? static_cast<double>(x[r * d + cj]) - mean[cj] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < PCA_T; ++rr) {
      const double av = a[rr][ty];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(av, b[rr][tx + 8 * q], acc[q]);
    }
  }
  const uint64_t i = static_cast<uint64_t>(ti) * PCA_T + ty;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint64_t j = static_cast<uint64_t>(tj) * PCA_T + tx + 8 * q;
    if (i < d && j < d) partial[(chunk * d + i) * d + j] = acc[q];
  }
}

__global__ void cov_reduce_kernel(const double* __restrict__ partial, uint64_t chunks, uint64_t dd,
                                  double* __restrict__ cov) {
  const uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= dd) return;
  double s = 0.0;
  for (uint64_t c = 0; c < chunks; ++c) s += partial[c * dd + e];
  cov[e] = s;
}

// out (n x k, f32) = scale * (x - mean) V for V (d x k, f32, row-major), k <= 128: 64 rows per block,
// d in slices of 32 staged in shared memory, f64 accumulation.
constexpr int PJ_ROWS = 64, PJ_D = 32, PJ_K = 128;
__global__ void __launch_bounds__(256) project_kernel(const float* __restrict__ x, uint64_t n, uint64_t d,
                                                      const double* __restrict__ mean, const float* __restrict__ V,
                                                      int k, float scale, float* __restrict__ out) {
  __shared__ float xs[PJ_ROWS][PJ_D + 1];
  __shared__ float vs[PJ_D][PJ_K];
  const uint64_t row0 = static_cast<uint64_t>(blockIdx.x) * PJ_ROWS;
  // thread t: rows (t / 4) + 64 * 0, columns (t % 4) + 4 q for q < k / 4 (rounded up)
  const int tr = threadIdx.x >> 2, tc = threadIdx.x & 3;
  double acc[PJ_K / 4];
#pragma unroll
  for (int q = 0; q < PJ_K / 4; ++q) acc[q] = 0.0;
  for (uint64_t c0 = 0; c0 < d; c0 += PJ_D) {
    __syncthreads();
    for (int e = threadIdx.x; e < PJ_ROWS * PJ_D; e += 256) {
      const int rr = e / PJ_D, cc = e % PJ_D;
      const uint64_t r = row0 + rr, c = c0 + cc;
      xs[rr][cc] = (r < n && c < d) ? static_cast<float>(static_cast<double>(x[r * d + c]) - mean[c]) : 0.0f;
    }
    for (int e = threadIdx.x; e < PJ_D * PJ_K; e += 256) {
      const int rr = e / PJ_K, cc = e % PJ_K;
      const uint64_t c = c0 + rr;
      vs[rr][cc] = (c < d && cc < k) ? V[c * k + cc] : 0.0f;
    }
    __syncthreads();
    for (int cc = 0; cc < PJ_D; ++cc) {
      const double xv = xs[tr][cc];
#pragma unroll
      for (int q = 0; q < PJ_K / 4; ++q) acc[q] = fma(xv, static_cast<double>(vs[cc][tc + 4 * q]), acc[q]);
    }
  }
  const uint64_t r = row0 + tr;
  if (r >= n) return;
#pragma unroll
  for (int q = 0; q < PJ_K / 4; ++q) {
    const int c = tc + 4 * q;
    if (c < k) out[r * k + c] = static_cast<float>(acc[q] * scale);
  }
}

// Cyclic Jacobi eigen-decomposition of a symmetric d x d matrix (row-major, f64): eigenvalues into w,
// eigenvectors as the columns of v.
void jacobi_eigen(std::vector<double>& a, int d, std::vector<double>& w, std::vector<double>& v) {
  v.assign(static_cast<size_t>(d) * d, 0.0);
  for (int i = 0; i < d; ++i) v[static_cast<size_t>(i) * d + i] = 1.0;
  auto A = [&](int i, int j) -> double& { return a[static_cast<size_t>(i) * d + j]; };
  double total = 0.0;
  for (double e : a) total += e * e;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < d; ++i)
      for (int j = i + 1; j < d; ++j) off += A(i, j) * A(i, j);
    if (off <= 1e-30 * total || off == 0.0) break;
    for (int p = 0; p < d - 1; ++p) {
      for (int q = p + 1; q < d; ++q) {
        const double apq = A(p, q);
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < d; ++k) {  // columns p, q
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < d; ++k) {  // rows p, q
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < d; ++k) {
          double* vk = &v[static_cast<size_t>(k) * d];
          const double vkp = vk[p], vkq = vk[q];
          vk[p] = c * vkp - s * vkq;
          vk[q] = s * vkp + c * vkq;
        }
      }
    }
  }
  w.resize(d);
  for (int i = 0; i < d; ++i) w[i] = A(i, i);
}

// Orthonormal columns (modified Gram-Schmidt) of a d x m matrix (row-major).
void orthonormalise(std::vector<double>& q, int d, int m) {
  for (int j = 0; j < m; ++j) {
    for (int i = 0; i < j; ++i) {
      double dot = 0.0;
      for (int r = 0; r < d; ++r) dot += q[static_cast<size_t>(r) * m + i] * q[static_cast<size_t>(r) * m + j];
      for (int r = 0; r < d; ++r) q[static_cast<size_t>(r) * m + j] -= dot * q[static_cast<size_t>(r) * m + i];
    }
    double nrm = 0.0;
    for (int r = 0; r < d; ++r) nrm += q[static_cast<size_t>(r) * m + j] * q[static_cast<size_t>(r) * m + j];
    nrm = std::sqrt(nrm);
    for (int r = 0; r < d; ++r) q[static_cast<size_t>(r) * m + j] = nrm > 0 ? q[static_cast<size_t>(r) * m + j] / nrm : 0.0;
  }
}

// The k leading eigenvectors of the symmetric d x d matrix a (columns of the returned d x k matrix,
// by descending eigenvalue, largest-magnitude entry positive).
std::vector<double> top_axes(std::vector<double>& a, int d, int k) {
  std::vector<double> vecs, w;  // d x m eigenvector block and its eigenvalues
  int m;
  if (d <= 160) {
    jacobi_eigen(a, d, w, vecs);
    m = d;
  } else {
    m = std::min(d, k + 24);
    std::vector<double> q(static_cast<size_t>(d) * m), t(static_cast<size_t>(d) * m);
    uint64_t state = 0x9E3779B97F4A7C15ull;  // fixed start: a splitmix64 stream in [-1, 1)
    for (auto& e : q) {
      state += 0x9E3779B97F4A7C15ull;
      uint64_t z = state;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      e = static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
    orthonormalise(q, d, m);
    for (int it = 0; it < 20; ++it) {
      std::fill(t.begin(), t.end(), 0.0);
      for (int r = 0; r < d; ++r)
        for (int l = 0; l < d; ++l) {
          const double arl = a[static_cast<size_t>(r) * d + l];
          const double* ql = &q[static_cast<size_t>(l) * m];
          double* tr = &t[static_cast<size_t>(r) * m];
          for (int j = 0; j < m; ++j) tr[j] += arl * ql[j];
        }
      q.swap(t);
      orthonormalise(q, d, m);
    }
    // Rayleigh-Ritz: the m x m projection q^T a q, its eigenvectors rotate q
    std::vector<double> aq(static_cast<size_t>(d) * m, 0.0), proj(static_cast<size_t>(m) * m, 0.0), z;
    for (int r = 0; r < d; ++r)
      for (int l = 0; l < d; ++l) {
        const double arl = a[static_cast<size_t>(r) * d + l];
        for (int j = 0; j < m; ++j) aq[static_cast<size_t>(r) * m + j] += arl * q[static_cast<size_t>(l) * m + j];
      }
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        double s = 0.0;
        for (int r = 0; r < d; ++r) s += q[static_cast<size_t>(r) * m + i] * aq[static_cast<size_t>(r) * m + j];
        proj[static_cast<size_t>(i) * m + j] = s;
      }
    for (int i = 0; i < m; ++i)  // symmetrise the rounding
      for (int j = i + 1; j < m; ++j) {
        const double s = 0.5 * (proj[static_cast<size_t>(i) * m + j] + proj[static_cast<size_t>(j) * m + i]);
        proj[static_cast<size_t>(i) * m + j] = proj[static_cast<size_t>(j) * m + i] = s;
      }
    jacobi_eigen(proj, m, w, z);
    vecs.assign(static_cast<size_t>(d) * m, 0.0);
    for (int r = 0; r < d; ++r)
      for (int j = 0; j < m; ++j) {
        double s = 0.0;
        for (int l = 0; l < m; ++l) s += q[static_cast<size_t>(r) * m + l] * z[static_cast<size_t>(l) * m + j];
        vecs[static_cast<size_t>(r) * m + j] = s;
      }
  }
  std::vector<int> order(m);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return w[p] > w[q]; });
  std::vector<double> V(static_cast<size_t>(d) * k);
  for (int j = 0; j < k; ++j) {
    const int col = order[j];
    int arg = 0;
    for (int r = 1; r < d; ++r)
      if (std::fabs(vecs[static_cast<size_t>(r) * m + col]) > std::fabs(vecs[static_cast<size_t>(arg) * m + col])) arg = r;
    const double sign = vecs[static_cast<size_t>(arg) * m + col] < 0 ? -1.0 : 1.0;
    for (int r = 0; r < d; ++r) V[static_cast<size_t>(r) * k + j] = sign * vecs[static_cast<size_t>(r) * m + col];
  }
  return V;
}

// out (n x k) = scale * x[:, :k] for x (n x w).
__global__ void leading_columns_kernel(const float* __restrict__ x, uint64_t n, uint64_t w, uint64_t k, float scale,
                                       float* __restrict__ out) {
  const uint64_t total = n * k;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t r = t / k, c = t - r * k;
    out[t] = __fmul_rn(x[r * w + c], scale);
  }
}

}  // namespace

void pca_top_axes(const double* cov, uint64_t d, uint64_t k, double* axes) {
  PM_REQUIRE(k >= 1 && k <= d && d <= 1024, PACMAP_ERR_UNSUPPORTED, "axes need 1 <= k <= d <= 1024");
  std::vector<double> a(cov, cov + d * d);
  const std::vector<double> V = top_axes(a, static_cast<int>(d), static_cast<int>(k));
  std::copy(V.begin(), V.end(), axes);
}

void leading_columns(Ctx& c, const float* d_x, uint64_t n, uint64_t w, uint64_t k, float scale, float* d_out) {
  if (!n || !k) return;
  leading_columns_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(n * k, 256), c.sm_count * 16ull)), 256, 0,
                           c.stream>>>(d_x, n, w, k, scale, d_out);
  PM_LAUNCHED();
}

void pca_project_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t k, float scale, float* d_out,
                        std::vector<float>* axes_out) {
  PM_REQUIRE(n > 0, PACMAP_ERR_EMPTY_ARRAY_MEAN, "Failed to calculate mean axis: the array is empty");
  PM_REQUIRE(k >= 1 && k <= static_cast<uint64_t>(PJ_K) && k <= d, PACMAP_ERR_UNSUPPORTED,
             "PCA supports at most 128 components and no more than the columns");
  PM_REQUIRE(d <= 1024, PACMAP_ERR_UNSUPPORTED, "PCA supports d <= 1024");
  // 1. means
  DevBuf<double> mpart(c, static_cast<uint64_t>(MEAN_BLOCKS) * d), mean(c, d);
  col_sum_partial_kernel<<<MEAN_BLOCKS, 256, 0, c.stream>>>(d_x, n, d, mpart.get());
  PM_LAUNCHED();
  col_mean_final_kernel<<<ceil_div(d, 256), 256, 0, c.stream>>>(mpart.get(), MEAN_BLOCKS, n, d, mean.get());
  PM_LAUNCHED();
  // 2. covariance (unnormalised: the axes do not depend on the scale)
  const uint64_t rpc = std::max<uint64_t>(16384, (n + PCA_MAX_CHUNKS - 1) / PCA_MAX_CHUNKS);
  const uint64_t chunks = (n + rpc - 1) / rpc, tiles = (d + PCA_T - 1) / PCA_T;
  DevBuf<double> part(c, chunks * d * d), cov(c, d * d);
  cov_partial_kernel<<<dim3(static_cast<unsigned>(tiles), static_cast<unsigned>(tiles), static_cast<unsigned>(chunks)),
                       256, 0, c.stream>>>(d_x, n, d, rpc, mean.get(), part.get());
  PM_LAUNCHED();
  cov_reduce_kernel<<<ceil_div(d * d, 256), 256, 0, c.stream>>>(part.get(), chunks, d * d, cov.get());
  PM_LAUNCHED();
  std::vector<double> a(d * d);
  PM_CUDA(cudaMemcpyAsync(a.data(), cov.get(), d * d * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  // 3. axes
  const std::vector<double> V64 = top_axes(a, static_cast<int>(d), static_cast<int>(k));
  std::vector<float> V(d * k);
  for (uint64_t e = 0; e < d * k; ++e) V[e] = static_cast<float>(V64[e]);
  if (axes_out) *axes_out = V;
  // 4. projection
  DevBuf<float> dV;
  upload(c, dV, V.data(), d * k);
  project_kernel<<<ceil_div(n, PJ_ROWS), 256, 0, c.stream>>>(d_x, n, d, mean.get(), dV.get(), static_cast<int>(k),
                                                            scale, d_out);
  PM_LAUNCHED();
}

}  // namespace pacmap
