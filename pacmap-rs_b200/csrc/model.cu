// The learned model on disk and the transform of new points (no reference analogue: the reference
// embeds only the points it was fitted on, README.md:165).
//
// A model is the MLP of the learned initialiser (mlp.cu), the preprocessing constants of its training
// data (preprocess_x's min, max and column means, src/lib.rs:485-511) and the per-dimension mean and
// standard deviation of the training embedding (the network predicts z-scored coordinates, the targets
// pacmap_mlp_train standardises). Transform = the same preprocessing with the stored constants, the
// network, and the inverse standardisation: new points land in the training embedding's coordinates.
//
// File format (little-endian):
//   "PACMAPML" | u32 version (1) | u32 hidden width (512) | u64 d | u64 dim | u64 parameter count |
//   f32 min | f32 max | f32 mean[d] | f32 target mean[dim] | f32 target std[dim] | f32 params[count] |
//   u64 FNV-1a 64 of every preceding byte.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"
#include "mlp.cuh"

namespace pacmap {
namespace {

constexpr char kMagic[8] = {'P', 'A', 'C', 'M', 'A', 'P', 'M', 'L'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kHidden = 512;
constexpr uint64_t kMaxD = 4096, kMaxDim = 16;

uint64_t fnv1a(const unsigned char* p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// x' = ((x - min) / max) - mean[c] in preprocess_x's three f32 roundings (src/lib.rs:500-511).
__global__ void apply_preprocess_kernel(const float* __restrict__ x, uint64_t n, uint64_t d, float mn, float mx,
                                        const float* __restrict__ mean, float* __restrict__ out) {
  const uint64_t total = n * d;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t c = t % d;
    out[t] = __fsub_rn(__fdiv_rn(__fsub_rn(x[t], mn), mx), mean[c]);
  }
}

// y = z * std + mean per dimension (ms: mean[dim] then std[dim]).
__global__ void destandardise_kernel(float* __restrict__ y, uint64_t n, uint64_t dim, const float* __restrict__ ms) {
  const uint64_t total = n * dim;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t c = t % dim;
    y[t] = __fadd_rn(__fmul_rn(y[t], ms[dim + c]), ms[c]);
  }
}

struct Writer {
  std::vector<unsigned char> buf;
  template <typename T>
  void put(const T& v) {
    const auto* p = reinterpret_cast<const unsigned char*>(&v);
    buf.insert(buf.end(), p, p + sizeof(T));
  }
  void put_f32(const float* p, uint64_t n) {
    const auto* b = reinterpret_cast<const unsigned char*>(p);
    buf.insert(buf.end(), b, b + n * sizeof(float));
  }
};

struct Reader {
  const std::vector<unsigned char>& buf;
  size_t pos = 0;
  template <typename T>
  T get() {
    PM_REQUIRE(pos + sizeof(T) <= buf.size(), PACMAP_ERR_MODEL_FILE, "model file is truncated");
    T v;
    std::memcpy(&v, buf.data() + pos, sizeof(T));
    pos += sizeof(T);
    return v;
  }
  void get_f32(float* out, uint64_t n) {
    PM_REQUIRE(pos + n * sizeof(float) <= buf.size(), PACMAP_ERR_MODEL_FILE, "model file is truncated");
    if (out) std::memcpy(out, buf.data() + pos, n * sizeof(float));
    pos += n * sizeof(float);
  }
};

}  // namespace

void model_target_stats(const float* y, uint64_t n, uint64_t dim, float* mean, float* sd) {
  // The standardisation pacmap_mlp_train applies to its targets (f64 sums, population std).
  for (uint64_t c = 0; c < dim; ++c) {
    double s = 0.0, s2 = 0.0;
    for (uint64_t i = 0; i < n; ++i) s += y[i * dim + c];
    const double mu = s / static_cast<double>(n);
    for (uint64_t i = 0; i < n; ++i) s2 += (y[i * dim + c] - mu) * (y[i * dim + c] - mu);
    mean[c] = static_cast<float>(mu);
    sd[c] = static_cast<float>(std::sqrt(s2 / static_cast<double>(n)) + 1e-30);
  }
}

void model_save(const char* path, uint64_t d, uint64_t dim, const float* params, float pre_min, float pre_max,
                const float* pre_mean, const float* t_mean, const float* t_std) {
  PM_REQUIRE(d >= 1 && d <= kMaxD && dim >= 1 && dim <= kMaxDim, PACMAP_ERR_UNSUPPORTED,
             "models support d <= 4096 and dim <= 16");
  const uint64_t count = mlp_param_count(d, dim);
  Writer w;
  w.buf.insert(w.buf.end(), kMagic, kMagic + 8);
  w.put(kVersion);
  w.put(kHidden);
  w.put(d);
  w.put(dim);
  w.put(count);
  w.put(pre_min);
  w.put(pre_max);
  w.put_f32(pre_mean, d);
  w.put_f32(t_mean, dim);
  w.put_f32(t_std, dim);
  w.put_f32(params, count);
  w.put(fnv1a(w.buf.data(), w.buf.size()));
  std::FILE* f = std::fopen(path, "wb");
  PM_REQUIRE(f != nullptr, PACMAP_ERR_MODEL_FILE, std::string("cannot open ") + path + " for writing");
  const size_t wrote = std::fwrite(w.buf.data(), 1, w.buf.size(), f);
  const int closed = std::fclose(f);
  PM_REQUIRE(wrote == w.buf.size() && closed == 0, PACMAP_ERR_MODEL_FILE, std::string("cannot write ") + path);
}

void model_load(const char* path, uint64_t* d_out, uint64_t* dim_out, float* params, float* pre_min, float* pre_max,
                float* pre_mean, float* t_mean, float* t_std) {
  std::FILE* f = std::fopen(path, "rb");
  PM_REQUIRE(f != nullptr, PACMAP_ERR_MODEL_FILE, std::string("cannot open ") + path);
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(f);
  PM_REQUIRE(buf.size() >= 8 + 8 && std::memcmp(buf.data(), kMagic, 8) == 0, PACMAP_ERR_MODEL_FILE,
             std::string(path) + " is not a PaCMAP model file");
  uint64_t stored;
  std::memcpy(&stored, buf.data() + buf.size() - 8, 8);
  PM_REQUIRE(fnv1a(buf.data(), buf.size() - 8) == stored, PACMAP_ERR_MODEL_FILE,
             std::string(path) + ": checksum mismatch (the file is damaged)");
  Reader r{buf, 8};
  const uint32_t version = r.get<uint32_t>(), hidden = r.get<uint32_t>();
  PM_REQUIRE(version == kVersion && hidden == kHidden, PACMAP_ERR_MODEL_FILE,
             std::string(path) + ": unsupported model version or hidden width");
  const uint64_t d = r.get<uint64_t>(), dim = r.get<uint64_t>(), count = r.get<uint64_t>();
  PM_REQUIRE(d >= 1 && d <= kMaxD && dim >= 1 && dim <= kMaxDim && count == mlp_param_count(d, dim),
             PACMAP_ERR_MODEL_FILE, std::string(path) + ": inconsistent model shape");
  const uint64_t body = 8 + 4 + 4 + 8 * 3 + 4 * (2 + d + 2 * dim + count) + 8;
  PM_REQUIRE(buf.size() == body, PACMAP_ERR_MODEL_FILE, std::string(path) + ": wrong file size for its shape");
  if (d_out) *d_out = d;
  if (dim_out) *dim_out = dim;
  const float mn = r.get<float>(), mx = r.get<float>();
  if (pre_min) *pre_min = mn;
  if (pre_max) *pre_max = mx;
  r.get_f32(pre_mean, d);
  r.get_f32(t_mean, dim);
  r.get_f32(t_std, dim);
  r.get_f32(params, count);
}

void destandardise_device(Ctx& c, float* d_y, uint64_t n, uint64_t dim, const float* t_mean, const float* t_std) {
  std::vector<float> ms(2 * dim);
  for (uint64_t k = 0; k < dim; ++k) {
    ms[k] = t_mean[k];
    ms[dim + k] = t_std[k];
  }
  DevBuf<float> dms;
  upload(c, dms, ms.data(), 2 * dim);
  const unsigned g = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n * dim, 256), c.sm_count * 16ull));
  destandardise_kernel<<<g, 256, 0, c.stream>>>(d_y, n, dim, dms.get());
  PM_LAUNCHED();
}

void transform_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t dim, const float* params,
                      float pre_min, float pre_max, const float* pre_mean, const float* t_mean, const float* t_std,
                      float* d_out) {
  if (n == 0) return;
  PM_REQUIRE(d >= 1 && d <= kMaxD && dim >= 1 && dim <= kMaxDim, PACMAP_ERR_UNSUPPORTED,
             "models support d <= 4096 and dim <= 16");
  DevBuf<float> xp(c, n * d), consts;
  upload(c, consts, pre_mean, d);
  std::vector<float> ms(2 * dim);
  for (uint64_t k = 0; k < dim; ++k) {
    ms[k] = t_mean[k];
    ms[dim + k] = t_std[k];
  }
  DevBuf<float> dms;
  upload(c, dms, ms.data(), 2 * dim);
  const unsigned g = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n * d, 256), c.sm_count * 16ull));
  apply_preprocess_kernel<<<g, 256, 0, c.stream>>>(d_x, n, d, pre_min, pre_max, consts.get(), xp.get());
  PM_LAUNCHED();
  mlp_apply_device(c, params, d, dim, xp.get(), n, d_out);
  const unsigned g2 = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n * dim, 256), c.sm_count * 16ull));
  destandardise_kernel<<<g2, 256, 0, c.stream>>>(d_out, n, dim, dms.get());
  PM_LAUNCHED();
  c.check_errors("transform");
}

}  // namespace pacmap
