// pacmap_preprocess_noalloc: preprocess_x (the same arithmetic as pacmap_preprocess) for callers that
// cannot allocate device memory -- e.g. a process whose device memory is owned by another framework's
// allocator or fixed by a budget, or a latency-critical loop that must not reach cudaMalloc/cudaFree
// (which can synchronise the device). The caller passes device input and output buffers and a stream;
// the only scratch (the total-order min/max keys and the column means) lives in the file-scope array
// below, which every GPU that loads the library holds until the process exits.
//
// The first call on a device looks up that array's device address (cudaGetSymbolAddress, with the
// device current) and caches it; make that first call before any stream capture. The address belongs to
// the device's primary context, so every call whose stream is not capturing looks it up again (after a
// cudaDeviceReset the cached one would be stale); a capturing call uses the cached one. The caller's
// current device is restored before the call returns. Every call shares the one array and leaves its
// contents behind: the min/max keys are reset at the start of each call, the means are overwritten.
// Calls that overlap on the GPU (two streams, or two host threads) race on the array and must be
// serialised by the caller.
#include <mutex>

#include "engine.cuh"

namespace pacmap {
namespace {

// Largest data dimension the scratch holds: 16,384 column means (64 KiB) + the two min/max keys.
constexpr uint64_t NOALLOC_MAX_D = 16384;

static __device__ __align__(256) uint32_t g_noalloc_scratch[4 + NOALLOC_MAX_D];

std::mutex g_noalloc_mutex;
uint32_t* g_noalloc_addr[64] = {};

__global__ void na_reset_keys_kernel(uint32_t* __restrict__ keys) {
  if (threadIdx.x == 0) {
    keys[0] = 0xFFFFFFFFu;
    keys[1] = 0u;
  }
}

__global__ void na_minmax_kernel(const float* __restrict__ x, uint64_t total, uint32_t* __restrict__ keys) {
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
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

constexpr int NA_COLS = 8, NA_ROWS = 512, NA_THREADS = 256;

// Column means in ndarray's sequential row order, reading min/max from the scratch keys.
__global__ void __launch_bounds__(NA_THREADS) na_colsum_kernel(const float* __restrict__ x, uint64_t n, uint64_t d,
                                                               const uint32_t* __restrict__ keys,
                                                               float* __restrict__ mean) {
  __shared__ float buf[2][NA_ROWS][NA_COLS];
  const float mn = key_to_float(keys[0]), mx = key_to_float(keys[1]);
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * NA_COLS;
  const int tid = threadIdx.x;
  const uint64_t nchunks = (n + NA_ROWS - 1) / NA_ROWS;
  auto stage = [&](uint64_t ch, int slot) {
    for (int e = tid - 32; e < NA_ROWS * NA_COLS; e += NA_THREADS - 32) {
      const int r = e / NA_COLS, cc = e % NA_COLS;
      const uint64_t row = ch * NA_ROWS + r, col = c0 + cc;
      float v = 0.0f;
      if (row < n && col < d) v = __fdiv_rn(__fsub_rn(x[row * d + col], mn), mx);
      buf[slot][r][cc] = v;
    }
  };
  if (tid >= 32) stage(0, 0);
  __syncthreads();
  float s = 0.0f;
  for (uint64_t ch = 0; ch < nchunks; ++ch) {
    if (tid >= 32 && ch + 1 < nchunks) stage(ch + 1, static_cast<int>((ch + 1) & 1));
    if (tid < NA_COLS) {
      const int rows = static_cast<int>((n - ch * NA_ROWS) < NA_ROWS ? (n - ch * NA_ROWS) : NA_ROWS);
      const int slot = static_cast<int>(ch & 1);
      for (int r = 0; r < rows; ++r) s = __fadd_rn(s, buf[slot][r][tid]);
    }
    __syncthreads();
  }
  if (tid < NA_COLS && c0 + tid < d) mean[c0 + tid] = __fdiv_rn(s, static_cast<float>(n));
}

__global__ void na_normalize_kernel(const float* __restrict__ x, uint64_t n, uint64_t d,
                                    const uint32_t* __restrict__ keys, const float* __restrict__ mean,
                                    float* __restrict__ out) {
  const float mn = key_to_float(keys[0]), mx = key_to_float(keys[1]);
  const uint64_t total = n * d;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const float y = __fdiv_rn(__fsub_rn(x[t], mn), mx);
    out[t] = __fsub_rn(y, mean[t % d]);
  }
}

// The scratch array's device address on `device` (that device current): looked up on a device's first
// call and on every call whose stream is not capturing (`refresh`), cached for capturing calls.
uint32_t* scratch_address(int device, bool refresh) {
  std::lock_guard<std::mutex> g(g_noalloc_mutex);
  if (g_noalloc_addr[device] && !refresh) return g_noalloc_addr[device];
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr)
    throw Fail{PACMAP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)};
  g_noalloc_addr[device] = static_cast<uint32_t*>(p);
  return g_noalloc_addr[device];
}

}  // namespace
}  // namespace pacmap

using namespace pacmap;

namespace {
// Puts the caller's current device back when the call returns, on every path.
struct RestoreDevice {
  int prev = -1;
  RestoreDevice() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
  }
  ~RestoreDevice() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" pacmap_status pacmap_preprocess_noalloc(const float* d_x, uint64_t n, uint64_t d, float* d_out,
                                                   void* stream, int32_t device) {
  RestoreDevice restore;
  try {
    PM_REQUIRE(d_x != nullptr && d_out != nullptr, PACMAP_ERR_INVALID_ARGUMENT, "NULL buffer");
    PM_REQUIRE(n * d > 0, PACMAP_ERR_EMPTY_ARRAY_MIN_MAX, "Failed to compute min or max of X: the array is empty");
    PM_REQUIRE(d <= NOALLOC_MAX_D, PACMAP_ERR_UNSUPPORTED,
               "pacmap_preprocess_noalloc supports at most " + std::to_string(NOALLOC_MAX_D) +
                   " columns (its fixed scratch holds that many column means)");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Fail{PACMAP_ERR_NO_DEVICE, "no CUDA device is visible"};
    }
    PM_REQUIRE(device >= 0 && device < count && device < 64, PACMAP_ERR_INVALID_ARGUMENT, "device not available");
    PM_CUDA(cudaSetDevice(device));
    int major = 0;
    PM_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    PM_REQUIRE(major == 10, PACMAP_ERR_NO_DEVICE, "device is not compute capability 10.x (sm_100)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PM_CUDA(cudaStreamIsCapturing(s, &cap));
    uint32_t* keys = scratch_address(device, cap == cudaStreamCaptureStatusNone);
    float* mean = reinterpret_cast<float*>(keys + 4);
    na_reset_keys_kernel<<<1, 32, 0, s>>>(keys);
    PM_LAUNCHED();
    int sms = 148;
    PM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const uint64_t total = n * d;
    na_minmax_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), sms * 8ull)), 256, 0, s>>>(
        d_x, total, keys);
    PM_LAUNCHED();
    na_colsum_kernel<<<ceil_div(d, NA_COLS), NA_THREADS, 0, s>>>(d_x, n, d, keys, mean);
    PM_LAUNCHED();
    na_normalize_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), sms * 16ull)), 256, 0, s>>>(
        d_x, n, d, keys, mean, d_out);
    PM_LAUNCHED();
    set_last_error("");
    return PACMAP_OK;
  } catch (const Fail& f) {
    set_last_error(f.msg);
    return f.code;
  }
}
