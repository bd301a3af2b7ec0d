// CPU oracle for the PaCMAP hot path -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 / OpenMP restatement of beamform/pacmap-rs v0.2.6 (crate `pacmap`), written from the
// reference's behaviour, used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
// the checker. The product (pacmap-rs_b200/) never links, loads or calls this file.
//
// Every function cites the reference file:line it follows. Floating-point semantics follow the
// reference's f32 path: separate IEEE mul/add/sub/div/sqrt (built with -ffp-contract=off), the
// 8-lane distance order of distance.rs:50-75, ndarray's sequential axis-0 sums, and f32 powi by
// square-and-multiply.
//
// Where the reference leaves an order unspecified (unstable sorts, rayon reductions), the oracle
// fixes one, and the GPU build matches it:
//   * kNN ties (knn.rs:167 par_sort_unstable_by) go to the lower neighbour index;
//   * scaled-distance ties (sampling.rs:410) go to the lower kNN column;
//   * MN candidate ties (sampling.rs:453) go to the earlier draw;
//   * the gradient (gradient.rs:53-70, rayon reduce) is summed sequentially in pair order.
//
// Parity status: the kNN, scale_dist, gradient, Adam and weight paths are pinned by the reference's
// own golden vectors (tests/test_oracle_golden.py). The random streams are NOT the reference's:
// rand 0.8.5 SmallRng / rand_distr 0.4.3 are replaced by a counter-based Philox4x32-10 stream
// (Salmon et al., SC'11) with the same rejection rule, so sampled pairs and Random init are
// "parity unpinned" against the reference and pinned only against this restatement.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int ORC_OK = 0;
constexpr int ORC_ERR_SAMPLE_SIZE = 1;
constexpr int ORC_ERR_INVALID_NN_SHAPE = 2;
constexpr int ORC_ERR_EMPTY_MEAN = 3;
constexpr int ORC_ERR_INVALID_NEIGHBOR_COUNT = 5;
constexpr int ORC_ERR_INVALID_FAR_COUNT = 6;
constexpr int ORC_ERR_EMPTY_MINMAX = 7;
constexpr int ORC_ERR_INVALID_ARGUMENT = 20;
constexpr int ORC_ERR_PAIR_INDEX = 21;
constexpr int ORC_ERR_SAMPLING = 22;

// f32::total_cmp as an order-preserving unsigned key (Rust core::f32::total_cmp).
inline uint32_t total_key(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// distance.rs:50-75 -- 8 f32 lane accumulators over chunks of 8, lanes summed 0..7, serial tail.
inline float ref_dist_sq(const float* a, const float* b, uint64_t d) {
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const uint64_t nc = d / 8;
  for (uint64_t c = 0; c < nc; ++c) {
    for (int l = 0; l < 8; ++l) {
      const float df = a[8 * c + l] - b[8 * c + l];
      acc[l] = acc[l] + df * df;
    }
  }
  float t = 0.0f;
  for (int l = 0; l < 8; ++l) t = t + acc[l];
  for (uint64_t i = nc * 8; i < d; ++i) {
    const float df = a[i] - b[i];
    t = t + df * df;
  }
  return t;
}
inline float ref_dist(const float* a, const float* b, uint64_t d) { return std::sqrt(ref_dist_sq(a, b, d)); }

// compiler-rt __powisf2, the lowering of Rust's f32::powi with a run-time exponent (adam.rs:47).
inline float powi_f32(float a, int b) {
  const bool recip = b < 0;
  float r = 1.0f;
  while (true) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}

// Rust `f as usize`: saturating, NaN -> 0.
inline uint64_t f32_as_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 18446744073709551616.0f) return UINT64_MAX;
  return static_cast<uint64_t>(f);
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
// ---------------------------------------------------------------------------------------------
inline void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Stream tags (counter word 3) separating the library's uses of one seed.
constexpr uint32_t TAG_SAMPLE = 0x53414D50u;  // 'SAMP': MN and FP draws of point i (one shared stream)
constexpr uint32_t TAG_INIT = 0x494E4954u;    // 'INIT': Random initialisation

// The per-point sampling stream: words w_0, w_1, ... with w_{4b+t} = philox(key=seed, ctr=(b, i_lo, i_hi, tag))[t].
struct PointStream {
  uint32_t k0, k1, c1, c2;
  uint32_t block = 0;
  uint32_t buf[4];
  int pos = 4;
  PointStream(uint64_t seed, uint64_t point)
      : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
        c1(static_cast<uint32_t>(point)), c2(static_cast<uint32_t>(point >> 32)) {}
  uint32_t next() {
    if (pos == 4) {
      const uint32_t ctr[4] = {block, c1, c2, TAG_SAMPLE};
      philox4x32_10(ctr, k0, k1, buf);
      ++block;
      pos = 0;
    }
    return buf[pos++];
  }
  // Uniform integer in [0, range): the widening-multiply rejection rule of rand 0.8.5
  // UniformInt<u32>::sample_single (zone = (range << lz(range)) - 1), fed by this stream.
  uint32_t uniform(uint32_t range) {
    const uint32_t zone = (range << __builtin_clz(range)) - 1u;
    while (true) {
      const uint32_t w = next();
      const uint64_t m = static_cast<uint64_t>(w) * range;
      if (static_cast<uint32_t>(m) <= zone) return static_cast<uint32_t>(m >> 32);
    }
  }
};

constexpr uint64_t SAMPLE_ATTEMPT_CAP = 1ull << 26;

// sampling.rs:37-61 `sample_fp`: n_samples distinct draws in [0, maximum), not `self_ind`, not in
// `reject` (strided view). Returns the number drawn, or -1 when the reference would loop forever
// (its `available` count over-states the distinct allowed values, e.g. duplicated rejects).
int sample_distinct(PointStream& s, uint32_t n_samples, uint32_t maximum, const uint32_t* reject,
                    uint64_t reject_stride, uint32_t n_reject, uint32_t self_ind, uint32_t* out) {
  bool self_in_reject = false;
  for (uint32_t t = 0; t < n_reject; ++t) self_in_reject |= (reject[t * reject_stride] == self_ind);
  uint64_t available = maximum;
  available = available > n_reject ? available - n_reject : 0;
  available = available > (self_in_reject ? 0u : 1u) ? available - (self_in_reject ? 0u : 1u) : 0;
  const uint32_t want = static_cast<uint32_t>(std::min<uint64_t>(n_samples, available));
  uint32_t cnt = 0;
  uint64_t attempts = 0;
  while (cnt < want) {
    if (++attempts > SAMPLE_ATTEMPT_CAP) return -1;
    const uint32_t j = s.uniform(maximum);
    if (j == self_ind) continue;
    bool dup = false;
    for (uint32_t t = 0; t < cnt && !dup; ++t) dup = (out[t] == j);
    for (uint32_t t = 0; t < n_reject && !dup; ++t) dup = (reject[t * reject_stride] == j);
    if (!dup) out[cnt++] = j;
  }
  return static_cast<int>(cnt);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------------------------------------
// Small exposed primitives (tests pin them against the reference's golden vectors).
// ------------------------------------------------------------------------------------------------
float orc_distance(const float* a, const float* b, uint64_t d) { return ref_dist(a, b, d); }
float orc_powi(float a, int b) { return powi_f32(a, b); }
uint32_t orc_total_key(float f) { return total_key(f); }

void orc_philox4x32_10(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
  philox4x32_10(ctr, k0, k1, out);
}

// The first `count` words of the sampling stream of `point`.
void orc_sample_stream(uint64_t seed, uint64_t point, uint32_t count, uint32_t* out) {
  PointStream s(seed, point);
  for (uint32_t t = 0; t < count; ++t) out[t] = s.next();
}

int orc_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
  return omp_get_max_threads();
#else
  (void)t;
  return 1;
#endif
}

// lib.rs:565-597 decide_num_pairs (f32 arithmetic, Rust round-half-away, saturating casts).
// override_k < 0 means "not overridden".
int orc_decide_num_pairs(uint64_t n, int64_t override_k, float mn_ratio, float fp_ratio, uint64_t* out3) {
  uint64_t k;
  if (override_k >= 0) {
    k = static_cast<uint64_t>(override_k);
  } else if (n <= 10000) {
    k = 10;
  } else {
    k = f32_as_usize(std::round(10.0f + 15.0f * (std::log10(static_cast<float>(n)) - 4.0f)));
  }
  const uint64_t n_mn = f32_as_usize(std::round(static_cast<float>(k) * mn_ratio));
  const uint64_t n_fp = f32_as_usize(std::round(static_cast<float>(k) * fp_ratio));
  out3[0] = k;
  out3[1] = n_mn;
  out3[2] = n_fp;
  if (k < 1) return ORC_ERR_INVALID_NEIGHBOR_COUNT;
  if (n_fp < 1) return ORC_ERR_INVALID_FAR_COUNT;
  return ORC_OK;
}

// lib.rs:485-511 preprocess_x (non-PCA branch): total_cmp min/max, x=(x-min), x=x/max (two f32 passes),
// column mean = ndarray mean_axis(Axis(0)) = sequential row-order sum / n, x -= mean.
int orc_preprocess(const float* x, uint64_t n, uint64_t d, float* out, float* out_min, float* out_max,
                   float* out_mean) {
  const uint64_t total = n * d;
  if (total == 0) return ORC_ERR_EMPTY_MINMAX;
  uint32_t kmin = total_key(x[0]), kmax = kmin;
  float vmin = x[0], vmax = x[0];
  for (uint64_t t = 1; t < total; ++t) {
    const uint32_t k = total_key(x[t]);
    if (k < kmin) { kmin = k; vmin = x[t]; }
    if (k >= kmax) { kmax = k; vmax = x[t]; }
  }
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < static_cast<int64_t>(total); ++t) {
    const float a = x[t] - vmin;
    out[t] = a / vmax;
  }
  std::vector<float> mean(d, 0.0f);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < static_cast<int64_t>(d); ++c) {
    float s = 0.0f;
    for (uint64_t r = 0; r < n; ++r) s = s + out[r * d + c];
    mean[c] = s / static_cast<float>(n);
  }
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < static_cast<int64_t>(n); ++r)
    for (uint64_t c = 0; c < d; ++c) out[r * d + c] = out[r * d + c] - mean[c];
  if (out_min) *out_min = vmin;
  if (out_max) *out_max = vmax;
  if (out_mean) std::memcpy(out_mean, mean.data(), d * sizeof(float));
  return ORC_OK;
}

// knn.rs:137-194 find_k_nearest_neighbors, per-row formulation: row i keeps the k'=min(k,n-1)
// smallest f32 distances to j != i, ordered by (distance, j). Identical to the reference's
// all-pairs + global sort + first-come fill when that sort breaks ties by (i, j).
int orc_knn_exact(const float* x, uint64_t n, uint64_t d, uint64_t k, uint32_t* idx, float* dist) {
  if (n == 0) return ORC_OK;
  const uint64_t kp = std::min<uint64_t>(k, n - 1);
  if (kp == 0) return ORC_OK;
#pragma omp parallel
  {
    std::vector<std::pair<uint64_t, uint32_t>> buf;  // (distance key, index)
    buf.reserve(n);
#pragma omp for schedule(dynamic, 8)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
      const uint64_t i = static_cast<uint64_t>(ii);
      buf.clear();
      for (uint64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        const float dd = ref_dist(x + i * d, x + j * d, d);
        buf.emplace_back((static_cast<uint64_t>(total_key(dd)) << 32) | j, static_cast<uint32_t>(j));
      }
      std::nth_element(buf.begin(), buf.begin() + (kp - 1), buf.end());
      std::sort(buf.begin(), buf.begin() + kp);
      for (uint64_t c = 0; c < kp; ++c) {
        idx[i * kp + c] = buf[c].second;
        const uint32_t key = static_cast<uint32_t>(buf[c].first >> 32);
        const uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
        float f;
        std::memcpy(&f, &u, 4);
        dist[i * kp + c] = f;
      }
    }
  }
  return ORC_OK;
}

// knn.rs:137-194 for a subset of query rows: out row q holds the k'=min(k,n-1) smallest f32
// distances from rows[q] to every j != rows[q], ordered by (distance, j) -- exactly row rows[q] of
// orc_knn_exact, without the O(n^2 d) full matrix. Rows go in groups of 8 against chunks of 2,048
// points, so each chunk is read from memory once per group; every row keeps its k' best (distance
// key, index) pairs in a max-heap.
int orc_knn_rows(const float* x, uint64_t n, uint64_t d, const uint32_t* rows, uint64_t m, uint64_t k, uint32_t* idx,
                 float* dist) {
  if (n == 0 || m == 0) return ORC_OK;
  for (uint64_t q = 0; q < m; ++q)
    if (rows[q] >= n) return ORC_ERR_INVALID_ARGUMENT;
  const uint64_t kp = std::min<uint64_t>(k, n - 1);
  if (kp == 0) return ORC_OK;
  constexpr uint64_t G = 8, CH = 2048;
  const int64_t groups = static_cast<int64_t>((m + G - 1) / G);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t g = 0; g < groups; ++g) {
    const uint64_t q0 = static_cast<uint64_t>(g) * G, q1 = std::min<uint64_t>(q0 + G, m);
    std::vector<std::vector<uint64_t>> heap(q1 - q0);
    for (auto& h : heap) h.reserve(kp + 1);
    for (uint64_t j0 = 0; j0 < n; j0 += CH) {
      const uint64_t j1 = std::min<uint64_t>(j0 + CH, n);
      for (uint64_t q = q0; q < q1; ++q) {
        const uint64_t i = rows[q];
        std::vector<uint64_t>& h = heap[q - q0];
        for (uint64_t j = j0; j < j1; ++j) {
          if (j == i) continue;
          const float dd = ref_dist(x + i * d, x + j * d, d);
          const uint64_t key = (static_cast<uint64_t>(total_key(dd)) << 32) | j;
          if (h.size() < kp) {
            h.push_back(key);
            std::push_heap(h.begin(), h.end());
          } else if (key < h.front()) {
            std::pop_heap(h.begin(), h.end());
            h.back() = key;
            std::push_heap(h.begin(), h.end());
          }
        }
      }
    }
    for (uint64_t q = q0; q < q1; ++q) {
      std::vector<uint64_t>& h = heap[q - q0];
      std::sort(h.begin(), h.end());
      for (uint64_t c = 0; c < kp; ++c) {
        idx[q * kp + c] = static_cast<uint32_t>(h[c] & 0xFFFFFFFFu);
        const uint32_t key = static_cast<uint32_t>(h[c] >> 32);
        const uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
        float f;
        std::memcpy(&f, &u, 4);
        dist[q * kp + c] = f;
      }
    }
  }
  return ORC_OK;
}

// knn.rs:149-191 restated literally: all n(n-1)/2 upper-triangle triples, one global sort by
// (distance, i, j), rows filled first come first served. Small n only (O(n^2) memory).
int orc_knn_exact_allpairs(const float* x, uint64_t n, uint64_t d, uint64_t k, uint32_t* idx, float* dist) {
  if (n == 0) return ORC_OK;
  const uint64_t kp = std::min<uint64_t>(k, n - 1);
  struct Tri { float dd; uint32_t i, j; };
  std::vector<Tri> tri;
  tri.reserve(n * (n - 1) / 2);
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t j = i + 1; j < n; ++j)
      tri.push_back({ref_dist(x + i * d, x + j * d, d), static_cast<uint32_t>(i), static_cast<uint32_t>(j)});
  std::sort(tri.begin(), tri.end(), [](const Tri& a, const Tri& b) {
    const uint32_t ka = total_key(a.dd), kb = total_key(b.dd);
    if (ka != kb) return ka < kb;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
  });
  std::vector<uint64_t> counts(n, 0);
  for (uint64_t t = 0; t < n * kp; ++t) { idx[t] = 0; dist[t] = 3.40282347e+38f; }
  for (const Tri& t : tri) {
    if (counts[t.i] < kp) { idx[t.i * kp + counts[t.i]] = t.j; dist[t.i * kp + counts[t.i]] = t.dd; ++counts[t.i]; }
    if (counts[t.j] < kp) { idx[t.j * kp + counts[t.j]] = t.i; dist[t.j * kp + counts[t.j]] = t.dd; ++counts[t.j]; }
  }
  return ORC_OK;
}

// neighbors.rs:79-84: sigma_i = mean(dist[i, start..end]) floored at 1e-10, start=min(3,k'-1),
// end=min(6,k'). ndarray's lane sum over <8 contiguous values is a sequential fold from 0.
void orc_sigma(const float* kd, uint64_t n, uint64_t kp, float* sig) {
  const uint64_t start = std::min<uint64_t>(3, kp > 0 ? kp - 1 : 0);
  const uint64_t end = std::min<uint64_t>(6, kp);
  for (uint64_t i = 0; i < n; ++i) {
    if (end <= start) { sig[i] = 1e-10f; continue; }
    float s = 0.0f;
    for (uint64_t c = start; c < end; ++c) s = s + kd[i * kp + c];
    const float m = s / static_cast<float>(end - start);
    sig[i] = std::fmax(m, 1e-10f);
  }
}

// distance.rs:27-37 scale_dist: d*d / (sigma_i * sigma_j).
void orc_scale_dist(const float* kd, const float* sig, const uint32_t* nbrs, uint64_t n, uint64_t kp, float* out) {
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t c = 0; c < kp; ++c) {
      const float dd = kd[i * kp + c];
      const float num = dd * dd;
      const float den = sig[i] * sig[nbrs[i * kp + c]];
      out[i * kp + c] = num / den;
    }
}

// sampling.rs:251-286 sample_neighbors_pair: per row, order the k' scaled distances by total_cmp
// (ties: lower column first), keep the first k, emit (i, neighbors[i, col]).
void orc_sample_neighbors_pair(const float* scaled, const uint32_t* nbrs, uint64_t n, uint64_t kp, uint64_t k,
                               uint32_t* pairs) {
#pragma omp parallel
  {
    std::vector<std::pair<uint32_t, uint32_t>> buf(kp);
#pragma omp for schedule(static)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
      const uint64_t i = static_cast<uint64_t>(ii);
      for (uint64_t c = 0; c < kp; ++c) buf[c] = {total_key(scaled[i * kp + c]), static_cast<uint32_t>(c)};
      std::sort(buf.begin(), buf.end());
      for (uint64_t j = 0; j < k; ++j) {
        pairs[(i * k + j) * 2 + 0] = static_cast<uint32_t>(i);
        pairs[(i * k + j) * 2 + 1] = nbrs[i * kp + buf[j].second];
      }
    }
  }
}

// sampling.rs:77-103 sample_fp_pair_deterministic with the Philox stream of point i: n_fp distinct
// partners, not i, not among pair_neighbors[i*k..(i+1)*k, 1]. Unfilled rows stay (0, 0).
int orc_sample_fp_pairs(const uint32_t* pair_neighbors, uint64_t n, uint64_t k, uint64_t n_fp, uint64_t seed,
                        uint32_t* out) {
  int err = ORC_OK;
  std::memset(out, 0, n * n_fp * 2 * sizeof(uint32_t));
#pragma omp parallel
  {
    std::vector<uint32_t> picks(n_fp);
#pragma omp for schedule(dynamic, 256)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
      const uint64_t i = static_cast<uint64_t>(ii);
      PointStream s(seed, i);
      const int cnt = sample_distinct(s, static_cast<uint32_t>(n_fp), static_cast<uint32_t>(n),
                                      pair_neighbors + (i * k) * 2 + 1, 2, static_cast<uint32_t>(k),
                                      static_cast<uint32_t>(i), picks.data());
      if (cnt < 0) {
#pragma omp atomic write
        err = ORC_ERR_SAMPLING;
        continue;
      }
      for (int t = 0; t < cnt; ++t) {
        out[(i * n_fp + t) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_fp + t) * 2 + 1] = picks[t];
      }
    }
  }
  return err;
}

// sampling.rs:118-142 + 296-313 sample_mn_pair_deterministic with the Philox stream of point i (the
// same stream the FP sampler of i starts from, as in the reference where both use seed+i): for each
// slot, 6 distinct candidates excluding i and earlier picks, then the 2nd smallest f32 distance.
// Fill entries (0.0, 0) stand in for missing candidates, as in the reference's [(0.0, 0); 6].
int orc_sample_mn_pairs(const float* x, uint64_t n, uint64_t d, uint64_t n_mn, uint64_t seed, uint32_t* out) {
  int err = ORC_OK;
  std::memset(out, 0, n * n_mn * 2 * sizeof(uint32_t));
#pragma omp parallel
  {
    std::vector<uint32_t> picks(n_mn + 1);
#pragma omp for schedule(dynamic, 256)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
      const uint64_t i = static_cast<uint64_t>(ii);
      PointStream s(seed, i);
      for (uint64_t j = 0; j < n_mn; ++j) {
        uint32_t cand[6];
        const int cnt = sample_distinct(s, 6, static_cast<uint32_t>(n), picks.data(), 1, static_cast<uint32_t>(j),
                                        static_cast<uint32_t>(i), cand);
        if (cnt < 0) {
#pragma omp atomic write
          err = ORC_ERR_SAMPLING;
          break;
        }
        std::pair<uint64_t, uint32_t> e[6];  // ((key << 3) | slot, index): stable by slot
        for (int t = 0; t < 6; ++t) {
          float dd = 0.0f;
          uint32_t id = 0;
          if (t < cnt) { id = cand[t]; dd = ref_dist(x + i * d, x + static_cast<uint64_t>(id) * d, d); }
          e[t] = {(static_cast<uint64_t>(total_key(dd)) << 3) | static_cast<uint64_t>(t), id};
        }
        std::sort(e, e + 6);
        picks[j] = e[1].second;
        out[(i * n_mn + j) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_mn + j) * 2 + 1] = e[1].second;
      }
    }
  }
  return err;
}

// weights.rs:52-81 find_weights -> (w_mn, w_nn, w_fp).
void orc_weights(uint64_t itr, uint64_t p1, uint64_t p2, float w_mn_init, float* w3) {
  if (itr < p1) {
    const float progress = static_cast<float>(itr) / static_cast<float>(p1);
    const float a = (1.0f - progress) * w_mn_init;
    const float b = progress * 3.0f;
    w3[0] = a + b;
    w3[1] = 2.0f;
    w3[2] = 1.0f;
  } else if (itr < p1 + p2) {
    w3[0] = 3.0f; w3[1] = 3.0f; w3[2] = 1.0f;
  } else {
    w3[0] = 0.0f; w3[1] = 1.0f; w3[2] = 1.0f;
  }
}

// adam.rs:45-47 (file lines) bias-corrected step size lr * sqrt(1 - b2^t) / (1 - b1^t), t = itr + 1.
float orc_lr_t(float lr, uint64_t itr) {
  const int t = static_cast<int>(itr + 1);
  const float s = std::sqrt(1.0f - powi_f32(0.999f, t));
  const float q = 1.0f - powi_f32(0.9f, t);
  return (lr * s) / q;
}

// gradient.rs:35-151 pacmap_grad, pairs summed sequentially (NN list, MN list, FP list, in row
// order). grad is (n+1) x dim with the loss at [n, 0]. Optional: grad64 (same sums in f64, from the
// f32 y) and abs_sum (per-element sum of |contribution|, for relative-error checks).
int orc_grad(const float* y, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn, const uint32_t* pmn,
             uint64_t n_mnp, const uint32_t* pfp, uint64_t n_fpp, float w_nn, float w_mn, float w_fp, float* grad,
             double* grad64, float* abs_sum) {
  std::memset(grad, 0, (n + 1) * dim * sizeof(float));
  if (grad64) std::memset(grad64, 0, (n + 1) * dim * sizeof(double));
  if (abs_sum) std::memset(abs_sum, 0, n * dim * sizeof(float));
  float loss = 0.0f;
  double loss64 = 0.0;
  std::vector<float> yij(dim);
  std::vector<double> yij64(dim);
  struct L { const uint32_t* p; uint64_t cnt; float w, dc, wc; bool fp; };
  const L lists[3] = {{pnn, n_nn, w_nn, 10.0f, 20.0f, false},
                      {pmn, n_mnp, w_mn, 10000.0f, 20000.0f, false},
                      {pfp, n_fpp, w_fp, 1.0f, 2.0f, true}};
  for (const L& l : lists) {
    for (uint64_t p = 0; p < l.cnt; ++p) {
      const uint64_t i = l.p[2 * p], j = l.p[2 * p + 1];
      if (i >= n || j >= n) return ORC_ERR_PAIR_INDEX;
      if (i == j) continue;
      float dij = 1.0f;
      double dij64 = 1.0;
      for (uint64_t c = 0; c < dim; ++c) {
        yij[c] = y[i * dim + c] - y[j * dim + c];
        dij = dij + yij[c] * yij[c];
        yij64[c] = static_cast<double>(y[i * dim + c]) - static_cast<double>(y[j * dim + c]);
        dij64 += yij64[c] * yij64[c];
      }
      float w1;
      double w164;
      if (l.fp) {
        loss = loss + l.w * (1.0f / (1.0f + dij));
        const float t = 1.0f + dij;
        w1 = l.w * (2.0f / (t * t));
        loss64 += static_cast<double>(l.w) / (1.0 + dij64);
        w164 = static_cast<double>(l.w) * 2.0 / ((1.0 + dij64) * (1.0 + dij64));
      } else {
        loss = loss + l.w * (dij / (l.dc + dij));
        const float t = l.dc + dij;
        w1 = l.w * (l.wc / (t * t));
        loss64 += static_cast<double>(l.w) * dij64 / (l.dc + dij64);
        w164 = static_cast<double>(l.w) * l.wc / ((l.dc + dij64) * (l.dc + dij64));
      }
      for (uint64_t c = 0; c < dim; ++c) {
        const float g = w1 * yij[c];
        if (l.fp) {
          grad[i * dim + c] = grad[i * dim + c] - g;
          grad[j * dim + c] = grad[j * dim + c] + g;
        } else {
          grad[i * dim + c] = grad[i * dim + c] + g;
          grad[j * dim + c] = grad[j * dim + c] - g;
        }
        if (grad64) {
          const double g64 = w164 * yij64[c];
          grad64[i * dim + c] += l.fp ? -g64 : g64;
          grad64[j * dim + c] += l.fp ? g64 : -g64;
        }
        if (abs_sum) {
          abs_sum[i * dim + c] += std::fabs(g);
          abs_sum[j * dim + c] += std::fabs(g);
        }
      }
    }
  }
  grad[n * dim] = loss;
  if (grad64) grad64[n * dim] = loss64;
  return ORC_OK;
}

// adam.rs:35-60 (file lines) update_embedding_adam, element-wise in f32.
void orc_adam(float* y, const float* grad, float* m, float* v, uint64_t count, float lr, uint64_t itr) {
  const float beta1 = 0.9f, beta2 = 0.999f;
  const float lr_t = orc_lr_t(lr, itr);
  const float a1 = 1.0f - beta1, a2 = 1.0f - beta2;
  for (uint64_t t = 0; t < count; ++t) {
    const float g = grad[t];
    m[t] = m[t] + a1 * (g - m[t]);
    v[t] = v[t] + a2 * (g * g - v[t]);
    const float num = lr_t * m[t];
    const float den = std::sqrt(v[t]) + 1e-7f;
    y[t] = y[t] - num / den;
  }
}

// lib.rs:753-766 Initialization::Value: (y - mean) * 0.0001 / std, mean = mean_axis(0) (sequential
// sum / n), std = sqrt(var_axis(0, ddof 0)) with ndarray's f32 Welford update (mul_add = fmaf).
int orc_init_value(const float* v, uint64_t n, uint64_t dim, float* y) {
  if (n == 0) return ORC_ERR_EMPTY_MEAN;
  std::vector<float> mean(dim, 0.0f), wmean(dim, 0.0f), ssq(dim, 0.0f), sd(dim);
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t c = 0; c < dim; ++c) mean[c] = mean[c] + v[i * dim + c];
  for (uint64_t c = 0; c < dim; ++c) mean[c] = mean[c] / static_cast<float>(n);
  for (uint64_t i = 0; i < n; ++i) {
    const float count = static_cast<float>(i + 1);
    for (uint64_t c = 0; c < dim; ++c) {
      const float xv = v[i * dim + c];
      const float delta = xv - wmean[c];
      wmean[c] = wmean[c] + delta / count;
      ssq[c] = std::fmaf(xv - wmean[c], delta, ssq[c]);
    }
  }
  for (uint64_t c = 0; c < dim; ++c) sd[c] = std::sqrt(ssq[c] / static_cast<float>(n));
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t c = 0; c < dim; ++c) {
      const float a = (v[i * dim + c] - mean[c]) * 0.0001f;
      y[i * dim + c] = a / sd[c];
    }
  return ORC_OK;
}

// Initialization::Random restated on the Philox stream (the reference's lib.rs:769-778 draws
// rand_distr's Normal(0,1) from SmallRng; that stream is not reproduced). Element t = i*dim + c:
// words (w0, w1) of philox(key=seed, ctr=(t>>1 lo, t>>1 hi, 0, 'INIT')), u1 = ((w0>>8)+1)/2^24,
// u2 = (w1>>8)/2^24, Box-Muller in f64: even t -> r cos(2 pi u2), odd t -> r sin(2 pi u2).
void orc_init_random(uint64_t n, uint64_t dim, uint64_t seed, float* y) {
  const uint64_t total = n * dim;
#pragma omp parallel for schedule(static)
  for (int64_t tt = 0; tt < static_cast<int64_t>(total); ++tt) {
    const uint64_t t = static_cast<uint64_t>(tt);
    const uint64_t q = t >> 1;
    const uint32_t ctr[4] = {static_cast<uint32_t>(q), static_cast<uint32_t>(q >> 32), 0u, TAG_INIT};
    uint32_t w[4];
    philox4x32_10(ctr, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), w);
    const double u1 = (static_cast<double>(w[0] >> 8) + 1.0) * (1.0 / 16777216.0);
    const double u2 = static_cast<double>(w[1] >> 8) * (1.0 / 16777216.0);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double a = 6.283185307179586476925286766559 * u2;
    y[t] = static_cast<float>((t & 1) ? r * std::sin(a) : r * std::cos(a));
  }
}

// lib.rs:736-843 pacmap(): m = v = 0, num_iters total iterations of weights -> grad -> Adam,
// snapshots (lib.rs:789-791, 830-836: slot 0 first holds the initial y; iteration itr writes the
// first slot whose index equals itr + 1). `y` holds the already-initialised embedding on entry and
// the result on exit. loss_out (optional) receives grad[n,0] per iteration.
int orc_optimize(float* y, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn, const uint32_t* pmn,
                 uint64_t n_mnp, const uint32_t* pfp, uint64_t n_fpp, float lr, uint64_t p1, uint64_t p2,
                 uint64_t p3, const uint64_t* snaps, uint64_t n_snaps, float* snap_out, float* loss_out) {
  const uint64_t cnt = n * dim;
  std::vector<float> m(cnt, 0.0f), v(cnt, 0.0f), grad((n + 1) * dim);
  if (n_snaps > 0 && snap_out) {
    std::memset(snap_out, 0, n_snaps * cnt * sizeof(float));
    std::memcpy(snap_out, y, cnt * sizeof(float));
  }
  const uint64_t total = p1 + p2 + p3;
  for (uint64_t itr = 0; itr < total; ++itr) {
    float w[3];
    orc_weights(itr, p1, p2, 1000.0f, w);
    const int rc = orc_grad(y, n, dim, pnn, n_nn, pmn, n_mnp, pfp, n_fpp, w[1], w[0], w[2], grad.data(), nullptr,
                            nullptr);
    if (rc != ORC_OK) return rc;
    if (loss_out) loss_out[itr] = grad[n * dim];
    orc_adam(y, grad.data(), m.data(), v.data(), cnt, lr, itr);
    if (n_snaps > 0 && snap_out) {
      for (uint64_t s = 0; s < n_snaps; ++s)
        if (snaps[s] == itr + 1) {
          std::memcpy(snap_out + s * cnt, y, cnt * sizeof(float));
          break;
        }
    }
  }
  return ORC_OK;
}

// One optimiser step from a given (y, m, v) state at iteration `itr`: the per-iteration parity
// harness. grad_out (optional) receives the (n+1) x dim gradient of that step.
// The reference's parallel optimiser loop, for the timed CPU baseline (the parity paths above stay
// sequential so that their sums have one fixed order). gradient.rs:35-74: the three pair lists cut into
// chunks of 128 * 1024 pairs; every chunk computes its contributions into its own zeroed (n+1) x dim
// array (process_pairs, gradient.rs:98-151) and the chunk arrays are folded and reduced across the
// worker threads (rayon par_bridge + reduce; here OpenMP threads fold in chunk order, then the thread
// accumulators are summed in thread order). adam.rs:35-60 with the element loop split across threads
// (Zip::par_for_each). The sums' order differs from the sequential oracle (as rayon's does between runs).
int orc_optimize_parallel(float* y, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn, const uint32_t* pmn,
                          uint64_t n_mnp, const uint32_t* pfp, uint64_t n_fpp, float lr, uint64_t p1, uint64_t p2,
                          uint64_t p3) {
  const uint64_t cnt = n * dim, gsz = (n + 1) * dim;
  constexpr uint64_t CHUNK = 128 * 1024;
  struct L { const uint32_t* p; uint64_t cnt; float dc, wc; bool fp; };
  const L lists[3] = {{pnn, n_nn, 10.0f, 20.0f, false}, {pmn, n_mnp, 10000.0f, 20000.0f, false},
                      {pfp, n_fpp, 1.0f, 2.0f, true}};
  std::vector<std::pair<int, uint64_t>> chunks;  // (list, first pair)
  for (int l = 0; l < 3; ++l)
    for (uint64_t a = 0; a < lists[l].cnt; a += CHUNK) chunks.push_back({l, a});
  for (int l = 0; l < 3; ++l)
    for (uint64_t q = 0; q < 2 * lists[l].cnt; ++q)
      if (lists[l].p[q] >= n) return ORC_ERR_PAIR_INDEX;
  std::vector<float> m(cnt, 0.0f), v(cnt, 0.0f), grad(gsz);
#ifdef _OPENMP
  const int nt = omp_get_max_threads();
#else
  const int nt = 1;
#endif
  std::vector<std::vector<float>> acc(nt, std::vector<float>(gsz));
  std::vector<float> tloss(nt);
  const uint64_t total = p1 + p2 + p3;
  for (uint64_t itr = 0; itr < total; ++itr) {
    float w3[3];
    orc_weights(itr, p1, p2, 1000.0f, w3);
    const float wl[3] = {w3[1], w3[0], w3[2]};
#pragma omp parallel
    {
#ifdef _OPENMP
      const int t = omp_get_thread_num();
#else
      const int t = 0;
#endif
      std::vector<float>& a = acc[t];
      std::fill(a.begin(), a.end(), 0.0f);
      float lsum = 0.0f;
      std::vector<float> g(gsz), yij(dim);
#pragma omp for schedule(dynamic, 1)
      for (int64_t ci = 0; ci < static_cast<int64_t>(chunks.size()); ++ci) {
        const L& l = lists[chunks[ci].first];
        const float w = wl[chunks[ci].first];
        const uint64_t b0 = chunks[ci].second, b1 = std::min<uint64_t>(b0 + CHUNK, l.cnt);
        std::fill(g.begin(), g.end(), 0.0f);  // process_pairs: Array2::zeros((n + 1, dim))
        float loss = 0.0f;
        for (uint64_t p = b0; p < b1; ++p) {
          const uint64_t i = l.p[2 * p], j = l.p[2 * p + 1];
          if (i == j) continue;
          float dij = 1.0f;
          for (uint64_t c = 0; c < dim; ++c) {
            yij[c] = y[i * dim + c] - y[j * dim + c];
            dij = dij + yij[c] * yij[c];
          }
          float w1;
          if (l.fp) {
            loss = loss + w * (1.0f / (1.0f + dij));
            const float tt = 1.0f + dij;
            w1 = w * (2.0f / (tt * tt));
          } else {
            loss = loss + w * (dij / (l.dc + dij));
            const float tt = l.dc + dij;
            w1 = w * (l.wc / (tt * tt));
          }
          for (uint64_t c = 0; c < dim; ++c) {
            const float gu = w1 * yij[c];
            if (l.fp) {
              g[i * dim + c] -= gu;
              g[j * dim + c] += gu;
            } else {
              g[i * dim + c] += gu;
              g[j * dim + c] -= gu;
            }
          }
        }
        for (uint64_t e = 0; e < gsz; ++e) a[e] += g[e];  // reduce: grad1 += &grad2
        lsum += loss;
      }
      tloss[t] = lsum;
    }
    std::fill(grad.begin(), grad.end(), 0.0f);
    float loss = 0.0f;
    for (int t = 0; t < nt; ++t) {
      for (uint64_t e = 0; e < gsz; ++e) grad[e] += acc[t][e];
      loss += tloss[t];
    }
    grad[n * dim] = loss;
    const int it = static_cast<int>(itr + 1);
    const float lr_t = lr * std::sqrt(1.0f - powi_f32(0.999f, it)) / (1.0f - powi_f32(0.9f, it));
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < static_cast<int64_t>(cnt); ++e) {
      const float gg = grad[e];
      m[e] = m[e] + (1.0f - 0.9f) * (gg - m[e]);
      v[e] = v[e] + (1.0f - 0.999f) * (gg * gg - v[e]);
      y[e] = y[e] - lr_t * m[e] / (std::sqrt(v[e]) + 1e-7f);
    }
  }
  return ORC_OK;
}

int orc_step(float* y, float* m, float* v, uint64_t n, uint64_t dim, const uint32_t* pnn, uint64_t n_nn,
             const uint32_t* pmn, uint64_t n_mnp, const uint32_t* pfp, uint64_t n_fpp, float lr, uint64_t p1,
             uint64_t p2, uint64_t itr, float* grad_out, double* grad64_out, float* abs_sum_out) {
  std::vector<float> grad((n + 1) * dim);
  float w[3];
  orc_weights(itr, p1, p2, 1000.0f, w);
  const int rc = orc_grad(y, n, dim, pnn, n_nn, pmn, n_mnp, pfp, n_fpp, w[1], w[0], w[2], grad.data(), grad64_out,
                          abs_sum_out);
  if (rc != ORC_OK) return rc;
  if (grad_out) std::memcpy(grad_out, grad.data(), (n + 1) * dim * sizeof(float));
  orc_adam(y, grad.data(), m, v, n * dim, lr, itr);
  return ORC_OK;
}

// neighbors.rs:56-108 generate_pairs (exact kNN branch, seeded sampling on the Philox stream).
// Output buffers: pnn (n*k x 2), pmn (n*n_mn x 2), pfp (n*n_fp x 2) with k = min(n_neighbors, n-1).
int orc_generate_pairs(const float* x, uint64_t n, uint64_t d, uint64_t n_neighbors, uint64_t n_mn, uint64_t n_fp,
                       uint64_t seed, uint32_t* pnn, uint32_t* pmn, uint32_t* pfp) {
  const uint64_t kp = std::min<uint64_t>(n_neighbors + 50, n - 1);
  const uint64_t k = std::min<uint64_t>(n_neighbors, n - 1);
  std::vector<uint32_t> nb(n * kp);
  std::vector<float> kd(n * kp), sig(n), sc(n * kp);
  int rc = orc_knn_exact(x, n, d, kp, nb.data(), kd.data());
  if (rc != ORC_OK) return rc;
  orc_sigma(kd.data(), n, kp, sig.data());
  orc_scale_dist(kd.data(), sig.data(), nb.data(), n, kp, sc.data());
  orc_sample_neighbors_pair(sc.data(), nb.data(), n, kp, k, pnn);
  rc = orc_sample_mn_pairs(x, n, d, n_mn, seed, pmn);
  if (rc != ORC_OK) return rc;
  return orc_sample_fp_pairs(pnn, n, k, n_fp, seed, pfp);
}

// ------------------------------------------------------------------------------------------------
// Quality metrics (no reference analogue; the library computes the same numbers on the GPU).
// ------------------------------------------------------------------------------------------------

// Mean fraction of each sampled point's `kk` nearest neighbours in the high-dimensional data that are
// also among its `kk` nearest neighbours in the embedding. Both neighbour sets use the reference's f32
// distance (distance.rs:50-75; in the embedding, dim < 8, that is the serial sum) ordered by
// (sqrt distance, index), as knn.rs ranks neighbours.
double orc_knn_preservation(const float* xh, uint64_t n, uint64_t d, const float* yl, uint64_t dim,
                            const uint32_t* sample, uint64_t n_sample, uint64_t kk) {
  double total = 0.0;
#pragma omp parallel
  {
    std::vector<std::pair<uint64_t, uint32_t>> bh, bl;
    bh.reserve(n);
    bl.reserve(n);
#pragma omp for schedule(dynamic, 4) reduction(+ : total)
    for (int64_t ss = 0; ss < static_cast<int64_t>(n_sample); ++ss) {
      const uint64_t i = sample[ss];
      bh.clear();
      bl.clear();
      for (uint64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        bh.emplace_back((static_cast<uint64_t>(total_key(ref_dist(xh + i * d, xh + j * d, d))) << 32) | j,
                        static_cast<uint32_t>(j));
        float s = 0.0f;
        for (uint64_t c = 0; c < dim; ++c) {
          const float df = yl[i * dim + c] - yl[j * dim + c];
          s = s + df * df;
        }
        bl.emplace_back((static_cast<uint64_t>(total_key(std::sqrt(s))) << 32) | j, static_cast<uint32_t>(j));
      }
      const uint64_t kq = std::min<uint64_t>(kk, bh.size());
      std::nth_element(bh.begin(), bh.begin() + (kq - 1), bh.end());
      std::nth_element(bl.begin(), bl.begin() + (kq - 1), bl.end());
      std::vector<uint32_t> a, b;
      for (uint64_t t = 0; t < kq; ++t) { a.push_back(bh[t].second); b.push_back(bl[t].second); }
      std::sort(a.begin(), a.end());
      std::sort(b.begin(), b.end());
      std::vector<uint32_t> inter;
      std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(inter));
      total += static_cast<double>(inter.size()) / static_cast<double>(kq);
    }
  }
  return n_sample ? total / static_cast<double>(n_sample) : 0.0;
}

// Fraction of triplets (i, j, l) whose order "j closer to i than l" agrees between the data and the
// embedding (same distance definitions as above).
double orc_triplet_accuracy(const float* xh, uint64_t d, const float* yl, uint64_t dim, const uint32_t* trip,
                            uint64_t n_trip) {
  uint64_t ok = 0;
#pragma omp parallel for reduction(+ : ok) schedule(static)
  for (int64_t t = 0; t < static_cast<int64_t>(n_trip); ++t) {
    const uint64_t i = trip[3 * t], j = trip[3 * t + 1], l = trip[3 * t + 2];
    const float hj = ref_dist_sq(xh + i * d, xh + j * d, d), hl = ref_dist_sq(xh + i * d, xh + l * d, d);
    float sj = 0.0f, sl = 0.0f;
    for (uint64_t c = 0; c < dim; ++c) {
      const float a = yl[i * dim + c] - yl[j * dim + c];
      const float b = yl[i * dim + c] - yl[l * dim + c];
      sj = sj + a * a;
      sl = sl + b * b;
    }
    ok += ((hj < hl) == (sj < sl)) ? 1u : 0u;
  }
  return n_trip ? static_cast<double>(ok) / static_cast<double>(n_trip) : 0.0;
}

// ------------------------------------------------------------------------------------------------
// Whole pipeline: lib.rs:294-367 fit_transform with Generate pairs (seeded) and Value or Random
// init. init_kind: 1 = Value (init_value n x dim), 2 = Random (seed). Writes n x dim.
// ------------------------------------------------------------------------------------------------
int orc_fit_transform(const float* x, uint64_t n, uint64_t d, uint64_t dim, int init_kind, const float* init_value,
                      uint64_t init_seed, float mn_ratio, float fp_ratio, int64_t override_k, uint64_t seed, float lr,
                      uint64_t p1, uint64_t p2, uint64_t p3, float* out) {
  if (n <= 1) return ORC_ERR_SAMPLE_SIZE;
  std::vector<float> xp(n * d);
  int rc = orc_preprocess(x, n, d, xp.data(), nullptr, nullptr, nullptr);
  if (rc != ORC_OK) return rc;
  uint64_t np[3];
  rc = orc_decide_num_pairs(n, override_k, mn_ratio, fp_ratio, np);
  if (rc != ORC_OK) return rc;
  const uint64_t k = std::min<uint64_t>(np[0], n - 1);
  std::vector<uint32_t> pnn(n * k * 2), pmn(n * np[1] * 2), pfp(n * np[2] * 2);
  rc = orc_generate_pairs(xp.data(), n, d, np[0], np[1], np[2], seed, pnn.data(), pmn.data(), pfp.data());
  if (rc != ORC_OK) return rc;
  if (init_kind == 1) {
    rc = orc_init_value(init_value, n, dim, out);
    if (rc != ORC_OK) return rc;
  } else if (init_kind == 2) {
    orc_init_random(n, dim, init_seed, out);
  } else {
    return ORC_ERR_INVALID_ARGUMENT;
  }
  return orc_optimize(out, n, dim, pnn.data(), n * k, pmn.data(), n * np[1], pfp.data(), n * np[2], lr, p1, p2, p3,
                      nullptr, 0, nullptr, nullptr);
}

}  // extern "C"
