// Shared device/host helpers of the B200 PaCMAP engine.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/pacmap.h"

namespace pacmap {

// ---------------------------------------------------------------------------------------------
// Status plumbing: every host-side stage returns a pacmap_status; a failure carries a message.
// ---------------------------------------------------------------------------------------------
struct Fail {
  pacmap_status code;
  std::string msg;
};

void set_last_error(const std::string& msg);
void count_launch(uint64_t k = 1);

#define PM_CUDA(expr)                                                                                        \
  do {                                                                                                       \
    cudaError_t e_ = (expr);                                                                                 \
    if (e_ != cudaSuccess) {                                                                                 \
      throw ::pacmap::Fail{e_ == cudaErrorMemoryAllocation ? PACMAP_ERR_OOM : PACMAP_ERR_CUDA,               \
                           std::string(#expr) + ": " + cudaGetErrorString(e_)};                              \
    }                                                                                                        \
  } while (0)

#define PM_LAUNCHED()                                                                                        \
  do {                                                                                                       \
    ::pacmap::count_launch();                                                                                \
    PM_CUDA(cudaGetLastError());                                                                             \
  } while (0)

#define PM_REQUIRE(cond, code, text)                                                                         \
  do {                                                                                                       \
    if (!(cond)) throw ::pacmap::Fail{(code), (text)};                                                       \
  } while (0)

// Device error word bits (kernels set them with atomicOr; the host checks after a stage).
enum DevErr : uint32_t {
  DEV_ERR_PAIR_INDEX = 1u << 0,    // a pair names a point >= n
  DEV_ERR_SAMPLING = 1u << 1,      // a sampler could not draw distinct partners
  DEV_ERR_TIMEOUT = 1u << 2,       // a bounded wait gave up
  DEV_ERR_CAPACITY = 1u << 3,      // a per-row buffer overflowed (the row is recomputed)
  DEV_ERR_INVARIANT = 1u << 4,     // any other internal check
};

inline unsigned ceil_div(uint64_t a, uint64_t b) { return static_cast<unsigned>((a + b - 1) / b); }

// ---------------------------------------------------------------------------------------------
// Exact f32 arithmetic (no contraction) and orders.
// ---------------------------------------------------------------------------------------------

// Rust f32::total_cmp as an order-preserving unsigned key.
__host__ __device__ __forceinline__ uint32_t total_key(float f) {
#ifdef __CUDA_ARCH__
  const uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key_to_float(uint32_t key) {
  return __uint_as_float((key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key);
}

// The reference's squared distance, src/distance.rs:50-75: 8 lane accumulators over chunks of 8
// (separately rounded sub, mul, add), lanes summed in order 0..7 from 0, then the serial tail.
__device__ __forceinline__ float ref_dist_sq(const float* __restrict__ a, const float* __restrict__ b, int d) {
  float acc[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) acc[l] = 0.0f;
  const int nc = d >> 3;
  for (int c = 0; c < nc; ++c) {
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const float df = __fsub_rn(a[8 * c + l], b[8 * c + l]);
      acc[l] = __fadd_rn(acc[l], __fmul_rn(df, df));
    }
  }
  float t = 0.0f;
#pragma unroll
  for (int l = 0; l < 8; ++l) t = __fadd_rn(t, acc[l]);
  for (int i = nc * 8; i < d; ++i) {
    const float df = __fsub_rn(a[i], b[i]);
    t = __fadd_rn(t, __fmul_rn(df, df));
  }
  return t;
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) and the per-point sampling stream.
// ---------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0, p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
#endif
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

constexpr uint32_t TAG_SAMPLE = 0x53414D50u;  // 'SAMP'
constexpr uint32_t TAG_INIT = 0x494E4954u;    // 'INIT'

// Words w_0, w_1, ... of point `point`: w_{4b+t} = philox(key = seed, ctr = (b, point_lo, point_hi, 'SAMP'))[t].
// The MN and FP samplers of a point both start this stream from word 0 (the reference seeds both
// with seed + i, src/sampling.rs:97,133).
struct PointStream {
  uint32_t k0, k1, c1, c2, block;
  uint32_t buf[4];
  int pos;
  __device__ __forceinline__ PointStream(uint64_t seed, uint64_t point)
      : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
        c1(static_cast<uint32_t>(point)), c2(static_cast<uint32_t>(point >> 32)), block(0), pos(4) {}
  __device__ __forceinline__ uint32_t next() {
    if (pos == 4) {
      philox4x32_10(block, c1, c2, TAG_SAMPLE, k0, k1, buf);
      ++block;
      pos = 0;
    }
    uint32_t w = buf[0];
    if (pos == 1) w = buf[1];
    if (pos == 2) w = buf[2];
    if (pos == 3) w = buf[3];
    ++pos;
    return w;
  }
  // rand 0.8.5 UniformInt<u32>::sample_single rule (zone = (range << lz(range)) - 1) on this stream.
  // Returns false when `budget` words ran out (the caller reports a sampling failure).
  __device__ __forceinline__ bool uniform(uint32_t range, uint32_t& out, uint64_t& budget) {
    const uint32_t zone = (range << __clz(range)) - 1u;
    while (budget > 0) {
      --budget;
      const uint32_t w = next();
      const uint32_t lo = w * range;
      if (lo <= zone) {
        out = __umulhi(w, range);
        return true;
      }
    }
    return false;
  }
};

// The same word sequence as PointStream, produced by a whole warp: lane L computes block base + L, so
// one Philox call per lane serves 128 draws, and word w of the batch comes from lane w / 4 by shuffle.
// Every lane must call next() / uniform() together (warp-uniform control flow).
struct WarpStream {
  uint32_t k0, k1, c1, c2, base;
  uint32_t buf[4];
  int pos;
  __device__ __forceinline__ WarpStream(uint64_t seed, uint64_t point)
      : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
        c1(static_cast<uint32_t>(point)), c2(static_cast<uint32_t>(point >> 32)), base(0), pos(128) {}
  __device__ __forceinline__ uint32_t next() {
    if (pos == 128) {
      philox4x32_10(base + (threadIdx.x & 31u), c1, c2, TAG_SAMPLE, k0, k1, buf);
      base += 32;
      pos = 0;
    }
    const int t = pos & 3;
    const uint32_t mine = t == 0 ? buf[0] : (t == 1 ? buf[1] : (t == 2 ? buf[2] : buf[3]));
    const uint32_t w = __shfl_sync(0xFFFFFFFFu, mine, pos >> 2);
    ++pos;
    return w;
  }
  __device__ __forceinline__ bool uniform(uint32_t range, uint32_t& out, uint64_t& budget) {
    const uint32_t zone = (range << __clz(range)) - 1u;
    while (budget > 0) {
      --budget;
      const uint32_t w = next();
      const uint32_t lo = w * range;
      if (lo <= zone) {
        out = __umulhi(w, range);
        return true;
      }
    }
    return false;
  }
};

constexpr uint64_t SAMPLE_ATTEMPT_CAP = 1ull << 26;

// ---------------------------------------------------------------------------------------------
// Packed two-wide f32 arithmetic (sm_100: one instruction for two round-to-nearest operations); a
// pair lives in one 64-bit register, element 0 in the low half.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t f32x2_pack(float2 v) {
  return static_cast<uint64_t>(__float_as_uint(v.x)) | (static_cast<uint64_t>(__float_as_uint(v.y)) << 32);
}
__device__ __forceinline__ float f32x2_lo(uint64_t v) { return __uint_as_float(static_cast<uint32_t>(v)); }
__device__ __forceinline__ float f32x2_hi(uint64_t v) { return __uint_as_float(static_cast<uint32_t>(v >> 32)); }
__device__ __forceinline__ uint64_t f32x2_sub(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f32x2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// ---------------------------------------------------------------------------------------------
// Warp helpers.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Ascending bitonic sort of 32 R 32-bit keys held in registers by one warp: element r * 32 + lane is
// v[r] of that lane. Partners closer than 32 elements are exchanged by shuffles, farther ones are registers
// of the same lane; no shared memory. Every lane must call it (warp-uniform R).
template <int R>
__device__ __forceinline__ void warp_sort_regs_u32(uint32_t (&v)[R]) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int size = 2; size <= 32 * R; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int rs = stride >> 5;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (r & rs) continue;
          const uint32_t e = static_cast<uint32_t>(r) * 32u + lane;
          const bool up = (e & static_cast<uint32_t>(size)) == 0u;
          const uint32_t a = v[r], b = v[r | rs];
          const bool sw = (a > b) == up;
          v[r] = sw ? b : a;
          v[r | rs] = sw ? a : b;
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t e = static_cast<uint32_t>(r) * 32u + lane;
          const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, v[r], stride);
          const bool up = (e & static_cast<uint32_t>(size)) == 0u;
          const bool lower = (lane & static_cast<uint32_t>(stride)) == 0u;
          v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
        }
      }
    }
  }
}

// The same network for 32 R 64-bit keys in registers.
template <int R>
__device__ __forceinline__ void warp_sort_regs_u64(uint64_t (&v)[R]) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int size = 2; size <= 32 * R; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int rs = stride >> 5;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (r & rs) continue;
          const uint32_t e = static_cast<uint32_t>(r) * 32u + lane;
          const bool up = (e & static_cast<uint32_t>(size)) == 0u;
          const uint64_t a = v[r], b = v[r | rs];
          const bool sw = (a > b) == up;
          v[r] = sw ? b : a;
          v[r | rs] = sw ? a : b;
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t e = static_cast<uint32_t>(r) * 32u + lane;
          const uint64_t o = __shfl_xor_sync(0xFFFFFFFFu, v[r], stride);
          const bool up = (e & static_cast<uint32_t>(size)) == 0u;
          const bool lower = (lane & static_cast<uint32_t>(stride)) == 0u;
          const bool take_min = lower == up;
          v[r] = ((o < v[r]) == take_min) ? o : v[r];
        }
      }
    }
  }
}

// In-place ascending bitonic sort of `len` (power of two) 64-bit keys in shared memory by one warp.
__device__ __forceinline__ void warp_bitonic_sort_u64(uint64_t* s, int len) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= len; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncwarp();
      for (int t = lane; t < (len >> 1); t += 32) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = ((i & size) == 0);
        const uint64_t a = s[i], b = s[j];
        if ((a > b) == up) {
          s[i] = b;
          s[j] = a;
        }
      }
    }
  }
  __syncwarp();
}

// Block-wide version (all threads of the block participate).
__device__ __forceinline__ void block_bitonic_sort_u64(uint64_t* s, int len) {
  for (int size = 2; size <= len; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int t = threadIdx.x; t < (len >> 1); t += blockDim.x) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = ((i & size) == 0);
        const uint64_t a = s[i], b = s[j];
        if ((a > b) == up) {
          s[i] = b;
          s[j] = a;
        }
      }
    }
  }
  __syncthreads();
}

__host__ __device__ __forceinline__ int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace pacmap
