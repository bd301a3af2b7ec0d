// K1 -- preprocess_x (src/lib.rs:485-511, non-PCA branch), bit-exact on the device:
//   min/max by f32::total_cmp            lib.rs:489-497
//   x = (x - min); x = x / max           lib.rs:500, 503 (two separately rounded f32 passes)
//   mean = mean_axis(Axis(0))            lib.rs:506-508 (ndarray: a sequential row-order f32 sum, then / n)
//   x -= mean                            lib.rs:511
// The column sum is an inherently serial chain per column (one rounded f32 add per row, in row
// order). A parallel pass first writes y = (x - min) / max into a buffer padded to 32 columns; then one
// warp per 32 columns runs the 32 chains (one lane per column) with the rows streamed into shared
// memory by a 6-stage TMA pipeline, so each chain runs at FADD latency; the division stays out of the
// serial warp. The centred output reads the same y.
#include <cstring>

#include "engine.cuh"
#include "tcgen05.cuh"

namespace pacmap {
namespace {

__global__ void minmax_keys_kernel(const float* __restrict__ x, uint64_t total, uint32_t* __restrict__ keys) {
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  // float4 path only for a 16-byte aligned base (device inputs may come from a caller).
  const uint64_t n4 = (reinterpret_cast<uintptr_t>(x) & 15u) ? 0 : total / 4;
  const float4* x4 = reinterpret_cast<const float4*>(x);
  for (uint64_t t = tid; t < n4; t += stride) {
    const float4 v = x4[t];
    const uint32_t a = total_key(v.x), b = total_key(v.y), cc = total_key(v.z), dd = total_key(v.w);
    kmin = min(kmin, min(min(a, b), min(cc, dd)));
    kmax = max(kmax, max(max(a, b), max(cc, dd)));
  }
  for (uint64_t t = n4 * 4 + tid; t < total; t += stride) {
    const uint32_t a = total_key(x[t]);
    kmin = min(kmin, a);
    kmax = max(kmax, a);
  }
  kmin = __reduce_min_sync(0xFFFFFFFFu, kmin);
  kmax = __reduce_max_sync(0xFFFFFFFFu, kmax);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&keys[0], kmin);
    atomicMax(&keys[1], kmax);
  }
}

constexpr int CQ_COLS = 32;    // columns per chain warp (one lane each)
constexpr int CQ_ROWS = 256;   // rows per TMA tile (32 KB)
constexpr int CQ_STAGES = 6;
static_assert(CQ_ROWS % 32 == 0, "the chain's full tiles run in steps of 32 rows");

// y = (x - sub) / div (two separately rounded f32 operations) into Y [n][dp], padding columns 0.
__global__ void scale_pad_kernel(const float* __restrict__ x, uint64_t n, uint64_t d, uint64_t dp, float sub,
                                 float div, float* __restrict__ Y) {
  const uint64_t total = n * dp;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t r = t / dp, c = t - r * dp;
    Y[t] = c < d ? __fdiv_rn(__fsub_rn(x[r * d + c], sub), div) : 0.0f;
  }
}

struct alignas(8) CqShared {
  uint64_t full[CQ_STAGES];
  uint64_t empty[CQ_STAGES];
  int abort_flag;
};

// mean[c] = (((0 + y_0c) + y_1c) + ... + y_(n-1)c) / n for the 32 columns of this block: warp 1 streams
// 256-row tiles of Y by TMA, warp 0 runs the chains (the next 16 rows are loaded while the current 16
// are added). Every wait is bounded.
__global__ void __launch_bounds__(64) colsum_chain_kernel(const __grid_constant__ CUtensorMap ymap, uint64_t n,
                                                          uint64_t d, float* __restrict__ mean,
                                                          uint32_t* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char cq_raw[];
  // aligned by offsetting the shared array itself: the chain's loads stay shared-memory loads
  float* buf = reinterpret_cast<float*>(cq_raw + ((128u - (smem_u32(cq_raw) & 127u)) & 127u));
  CqShared* sh = reinterpret_cast<CqShared*>(buf + CQ_STAGES * CQ_ROWS * CQ_COLS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = blockIdx.x * CQ_COLS;
  const uint64_t ntiles = (n + CQ_ROWS - 1) / CQ_ROWS;
  if (threadIdx.x == 0) {
    for (int s = 0; s < CQ_STAGES; ++s) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 1);
    }
    sh->abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  volatile int* abort_flag = &sh->abort_flag;
  if (warp == 1) {
    if (lane == 0) {
      uint64_t issued = 0;
      for (uint64_t t = 0; t < ntiles; ++t) {
        const int s = static_cast<int>(t % CQ_STAGES);
        if (t >= CQ_STAGES && !mbar_wait(&sh->empty[s], static_cast<uint32_t>(((t / CQ_STAGES) + 1) & 1), abort_flag))
          break;
        mbar_expect_tx(&sh->full[s], CQ_ROWS * CQ_COLS * 4);
        tma_load_2d(buf + s * CQ_ROWS * CQ_COLS, &ymap, &sh->full[s], c0, static_cast<int>(t * CQ_ROWS));
        issued = t + 1;
      }
      if (issued < ntiles) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      // every issued load has landed before the block exits
      for (uint64_t t = (issued > CQ_STAGES ? issued - CQ_STAGES : 0); t < issued; ++t) {
        const uint64_t t0 = globaltimer();
        while (!mbar_try_wait(&sh->full[t % CQ_STAGES], static_cast<uint32_t>((t / CQ_STAGES) & 1)) &&
               globaltimer() - t0 < WAIT_LIMIT_NS) {
        }
      }
    }
    return;
  }
  float s = 0.0f;
  for (uint64_t t = 0; t < ntiles; ++t) {
    const int st = static_cast<int>(t % CQ_STAGES);
    if (!mbar_wait(&sh->full[st], static_cast<uint32_t>((t / CQ_STAGES) & 1), abort_flag)) {
      if (lane == 0) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      return;
    }
    const float* b = buf + st * CQ_ROWS * CQ_COLS + lane;
    const int rows = static_cast<int>(n - t * CQ_ROWS < CQ_ROWS ? n - t * CQ_ROWS : CQ_ROWS);
    if (rows == CQ_ROWS) {
      // a full tile: two register sets in turn, one loaded while the other is added (no copies)
      float A[16], B[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) A[q] = b[q * CQ_COLS];
#pragma unroll
      for (int r = 0; r < CQ_ROWS; r += 32) {
#pragma unroll
        for (int q = 0; q < 16; ++q) B[q] = b[(r + 16 + q) * CQ_COLS];
#pragma unroll
        for (int q = 0; q < 16; ++q) s = __fadd_rn(s, A[q]);
        if (r + 32 < CQ_ROWS) {
#pragma unroll
          for (int q = 0; q < 16; ++q) A[q] = b[(r + 32 + q) * CQ_COLS];
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) s = __fadd_rn(s, B[q]);
      }
    } else {
      for (int r = 0; r < rows; ++r) s = __fadd_rn(s, b[r * CQ_COLS]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sh->empty[st]);
  }
  if (c0 + lane < static_cast<int>(d)) mean[c0 + lane] = __fdiv_rn(s, static_cast<float>(n));
}

// out = y - mean (lib.rs:511); y may be `out` itself (same pitch), each element read then written by
// one thread.
__global__ void normalize_center_kernel(const float* Y, uint64_t n, uint64_t d, uint64_t dp,
                                        const float* __restrict__ mean, float* out) {
  const uint64_t total = n * d;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t r = t / d, c = t - r * d;
    out[t] = __fsub_rn(Y[r * dp + c], mean[c]);
  }
}

// One thread per row: the norm as ref_dist_sq(row, 0) (8 lane sums over chunks of 8 in order, the lanes
// summed in order, then the tail), then every element divided by it.
__global__ void normalize_rows_kernel(float* __restrict__ x, uint64_t n, int d) {
  const uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float* row = x + r * d;
  float acc[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) acc[l] = 0.0f;
  const int nc = d >> 3;
  for (int ch = 0; ch < nc; ++ch) {
#pragma unroll
    for (int l = 0; l < 8; ++l) acc[l] = __fadd_rn(acc[l], __fmul_rn(row[8 * ch + l], row[8 * ch + l]));
  }
  float t = 0.0f;
#pragma unroll
  for (int l = 0; l < 8; ++l) t = __fadd_rn(t, acc[l]);
  for (int e = nc * 8; e < d; ++e) t = __fadd_rn(t, __fmul_rn(row[e], row[e]));
  const float nrm = __fsqrt_rn(t);
  if (!(nrm > 0.0f)) return;
  for (int e = 0; e < d; ++e) row[e] = __fdiv_rn(row[e], nrm);
}

}  // namespace

void normalize_rows_device(Ctx& c, float* d_x, uint64_t n, uint64_t d) {
  if (!n || !d) return;
  normalize_rows_kernel<<<ceil_div(n, 256), 256, 0, c.stream>>>(d_x, n, static_cast<int>(d));
  PM_LAUNCHED();
}

// y = (x - sub) / div with pitch dp = d rounded up to 4 floats (the TMA stride rule), written into
// `dst` when that pitch is d and dst is 16-byte aligned (no scratch at all), else into Y; then the
// sequential column means of y (the 32-column TMA boxes zero-fill columns beyond dp). Returns y.
const float* scaled_column_means(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float sub, float div, float* dst,
                                 DevBuf<float>& Y, float* d_mean, uint64_t& dp_out) {
  const uint64_t dp = (d + 3) / 4 * 4;
  float* y = dst;
  if (!(dst && dp == d && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0)) {
    Y.alloc(c, n * dp);
    y = Y.get();
  }
  const unsigned g = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n * dp, 256), c.sm_count * 16ull));
  scale_pad_kernel<<<g, 256, 0, c.stream>>>(d_x, n, d, dp, sub, div, y);
  PM_LAUNCHED();
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(dp), static_cast<cuuint64_t>(n)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(dp) * 4};
  const cuuint32_t box[2] = {CQ_COLS, CQ_ROWS};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult cr = detail::get_encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, y, dims, strides, box, estr,
                                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PM_REQUIRE(cr == CUDA_SUCCESS, PACMAP_ERR_CUDA, "cuTensorMapEncodeTiled (column sums) failed: " + std::to_string(cr));
  const size_t smem = 128 + static_cast<size_t>(CQ_STAGES) * CQ_ROWS * CQ_COLS * 4 + sizeof(CqShared);
  PM_CUDA(cudaFuncSetAttribute(colsum_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  colsum_chain_kernel<<<static_cast<unsigned>(ceil_div(d, static_cast<uint64_t>(CQ_COLS))), 64, smem, c.stream>>>(
      map, n, d, d_mean, c.d_err);
  PM_LAUNCHED();
  dp_out = dp;
  return y;
}

void column_mean_seq(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float sub, float div, float* d_mean) {
  DevBuf<float> Y;
  uint64_t dp = 0;
  scaled_column_means(c, d_x, n, d, sub, div, nullptr, Y, d_mean, dp);
}

void preprocess_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float* d_out, float* h_min, float* h_max,
                       float* d_mean) {
  const uint64_t total = n * d;
  PM_REQUIRE(total > 0, PACMAP_ERR_EMPTY_ARRAY_MIN_MAX, "Failed to compute min or max of X: the array is empty");
  DevBuf<uint32_t> keys(c, 2);
  const uint32_t init[2] = {0xFFFFFFFFu, 0u};
  PM_CUDA(cudaMemcpyAsync(keys.get(), init, sizeof(init), cudaMemcpyHostToDevice, c.stream));
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div(total / 4 + 1, 256), c.sm_count * 8ull));
  minmax_keys_kernel<<<grid, 256, 0, c.stream>>>(d_x, total, keys.get());
  PM_LAUNCHED();
  uint32_t hk[2];
  PM_CUDA(cudaMemcpyAsync(hk, keys.get(), sizeof(hk), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  auto decode = [](uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
  };
  const float mn = decode(hk[0]), mx = decode(hk[1]);
  if (h_min) *h_min = mn;
  if (h_max) *h_max = mx;
  DevBuf<float> mean_local;
  float* mean = d_mean;
  if (!mean) {
    mean_local.alloc(c, d);
    mean = mean_local.get();
  }
  DevBuf<float> Y;
  uint64_t dp = 0;
  const float* y = scaled_column_means(c, d_x, n, d, mn, mx, d_out, Y, mean, dp);  // y is d_out when d % 4 == 0
  const unsigned g2 = static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), c.sm_count * 16ull));
  normalize_center_kernel<<<g2, 256, 0, c.stream>>>(y, n, d, dp, mean, d_out);
  PM_LAUNCHED();
}

}  // namespace pacmap
