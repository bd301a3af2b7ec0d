// K1 -- preprocess_x (src/lib.rs:485-511, non-PCA branch), bit-exact on the device:
//   min/max by f32::total_cmp            lib.rs:489-497
//   x = (x - min); x = x / max           lib.rs:500, 503 (two separately rounded f32 passes)
//   mean = mean_axis(Axis(0))            lib.rs:506-508 (ndarray: a sequential row-order f32 sum, then / n)
//   x -= mean                            lib.rs:511
// The column sum is an inherently serial chain per column; it runs one lane per column with the rows
// streamed through shared memory by the other warps of the block, so the chain runs at FADD latency.
#include "engine.cuh"

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

constexpr int CS_COLS = 8;      // columns per block (one summing lane each)
constexpr int CS_ROWS = 512;    // rows per staged chunk
constexpr int CS_THREADS = 256; // warp 0 sums, warps 1..7 stage

__global__ void __launch_bounds__(CS_THREADS) colsum_seq_kernel(const float* __restrict__ x, uint64_t n,
                                                                uint64_t d, float sub, float div,
                                                                float* __restrict__ mean) {
  __shared__ float buf[2][CS_ROWS][CS_COLS];
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * CS_COLS;
  const int tid = threadIdx.x;
  const uint64_t nchunks = (n + CS_ROWS - 1) / CS_ROWS;
  auto stage = [&](uint64_t ch, int slot) {
    // warps 1..7 load rows [ch*R, ch*R + R) x columns [c0, c0 + 8), applying (v - sub) / div.
    for (int e = tid - 32; e < CS_ROWS * CS_COLS; e += CS_THREADS - 32) {
      const int r = e / CS_COLS, cc = e % CS_COLS;
      const uint64_t row = ch * CS_ROWS + r, col = c0 + cc;
      float v = 0.0f;
      if (row < n && col < d) v = __fdiv_rn(__fsub_rn(x[row * d + col], sub), div);
      buf[slot][r][cc] = v;
    }
  };
  if (tid >= 32) stage(0, 0);
  __syncthreads();
  float s = 0.0f;
  for (uint64_t ch = 0; ch < nchunks; ++ch) {
    if (tid >= 32 && ch + 1 < nchunks) stage(ch + 1, static_cast<int>((ch + 1) & 1));
    if (tid < CS_COLS) {
      const int rows = static_cast<int>((n - ch * CS_ROWS) < CS_ROWS ? (n - ch * CS_ROWS) : CS_ROWS);
      const int slot = static_cast<int>(ch & 1);
      int r = 0;
      for (; r + 16 <= rows; r += 16) {  // loads run ahead of the serial add chain
        float t[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) t[q] = buf[slot][r + q][tid];
#pragma unroll
        for (int q = 0; q < 16; ++q) s = __fadd_rn(s, t[q]);
      }
      for (; r < rows; ++r) s = __fadd_rn(s, buf[slot][r][tid]);
    }
    __syncthreads();
  }
  if (tid < CS_COLS && c0 + tid < d) mean[c0 + tid] = __fdiv_rn(s, static_cast<float>(n));
}

__global__ void normalize_center_kernel(const float* __restrict__ x, uint64_t n, uint64_t d, float mn, float mx,
                                        const float* __restrict__ mean, float* __restrict__ out) {
  const uint64_t total = n * d;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const float y = __fdiv_rn(__fsub_rn(x[t], mn), mx);
    out[t] = __fsub_rn(y, mean[t % d]);
  }
}

}  // namespace

void column_mean_seq(Ctx& c, const float* d_x, uint64_t n, uint64_t d, float sub, float div, float* d_mean) {
  colsum_seq_kernel<<<ceil_div(d, CS_COLS), CS_THREADS, 0, c.stream>>>(d_x, n, d, sub, div, d_mean);
  PM_LAUNCHED();
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
  column_mean_seq(c, d_x, n, d, mn, mx, mean);
  const unsigned g2 = static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), c.sm_count * 16ull));
  normalize_center_kernel<<<g2, 256, 0, c.stream>>>(d_x, n, d, mn, mx, mean, d_out);
  PM_LAUNCHED();
}

}  // namespace pacmap
