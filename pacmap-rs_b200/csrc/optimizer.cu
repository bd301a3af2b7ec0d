// The optimiser -- src/lib.rs:736-843 (pacmap), src/gradient.rs:35-151, src/adam.rs:35-60 (file lines),
// src/weights.rs:52-81.
//
// K7 build_csr: every pair (i, j), i != j, of the three lists becomes two entries -- partner j in the
//    segment (i, type) and partner i in the segment (j, type) -- via a counting sort, then each segment
//    is sorted by partner. When the lists are grouped by point (the generated ones are), a mid-near or
//    far segment is point i's own partners in pair order followed by the points that drew i, sorted:
//    only that second part is placed by atomics and sorted (a neighbour segment is sorted whole). A pair's contribution to each endpoint is bit-identical whichever endpoint
//    lists it (the squared distance and the weight use |y_i - y_j| only), so the sorted segments fix
//    one deterministic summation order with no floating-point atomics. (The reference's rayon reduce,
//    gradient.rs:53-70, has no fixed order at all.)
// K8 grad_adam_kernel: one group of G = 8 lanes per point sums its segments (NN c=10, MN c=10000, FP
//    repulsive c=1, exactly the per-pair f32 arithmetic of gradient.rs:120-147), reduces across the
//    group in a fixed butterfly, and applies the Adam step (adam.rs:45-57) to that point at once:
//    y is ping-ponged between two buffers because other points read y_j during the iteration.
//    Phase 3 has w_mn = 0: the MN segments are skipped (0 * finite = 0 adds nothing).
// K9 optimize_device: all iterations are captured into one CUDA graph (one kernel node per iteration,
//    snapshot copies as memcpy nodes); the per-iteration (w_nn, w_mn, w_fp, lr_t) schedule lives in a
//    device table computed with the reference's f32 formulas.
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>

#include "engine.cuh"

namespace pacmap {
namespace {

// ------------------------------------------------------------------------------------------------
// K7: CSR build
// ------------------------------------------------------------------------------------------------
__global__ void csr_count_kernel(const uint32_t* __restrict__ pairs, uint64_t P, int type, uint64_t n,
                                 uint32_t* __restrict__ cnt, uint32_t* __restrict__ err) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += stride) {
    const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
    if (a >= n || b >= n) {
      atomicOr(err, DEV_ERR_PAIR_INDEX);
      continue;
    }
    if (a == b) continue;
    atomicAdd(&cnt[static_cast<uint64_t>(a) * 3 + type], 1u);
    atomicAdd(&cnt[static_cast<uint64_t>(b) * 3 + type], 1u);
  }
}

__global__ void csr_fill_kernel(const uint32_t* __restrict__ pairs, uint64_t P, int type, uint64_t n,
                                uint32_t* __restrict__ cursor, uint32_t* __restrict__ col) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += stride) {
    const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
    if (a >= n || b >= n || a == b) continue;
    col[atomicAdd(&cursor[static_cast<uint64_t>(a) * 3 + type], 1u)] = b;
    col[atomicAdd(&cursor[static_cast<uint64_t>(b) * 3 + type], 1u)] = a;
  }
}

// The generated pair lists hold each point's pairs together (rows i*k .. i*k + k - 1 start with i). Then
// a segment's forward entries (partners of its own pairs) are written in pair order without atomics, and
// only the reverse entries (points that drew it) are placed by atomics and sorted.
__global__ void grouped_check_kernel(const uint32_t* __restrict__ pairs, uint64_t P, uint32_t k,
                                     uint32_t* __restrict__ flag) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  bool ok = true;
  for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += stride)
    ok = ok && pairs[2 * p] == static_cast<uint32_t>(p / k);
  if (!__all_sync(0xFFFFFFFFu, ok) && (threadIdx.x & 31) == 0) *flag = 0u;
}

// Forward counts of grouped lists: segment (i, type) gets the partners j != i of point i's k pairs. One
// warp per point, its pairs read in coalesced chunks of 32.
__global__ void __launch_bounds__(256) csr_fwd_count_kernel(const uint32_t* __restrict__ pairs, uint64_t n,
                                                            uint32_t k, int type, uint32_t* __restrict__ fwd,
                                                            uint32_t* __restrict__ cnt, uint32_t* __restrict__ err) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31;
  if (i >= n) return;
  uint32_t c = 0;
  bool bad = false;
  for (uint32_t q = lane; q < k; q += 32) {
    const uint32_t j = pairs[2 * (i * k + q) + 1];
    bad |= j >= n;
    c += (j < n && j != i) ? 1u : 0u;
  }
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(err, DEV_ERR_PAIR_INDEX);
  if (lane == 0) {
    fwd[i * 3 + type] = c;
    cnt[i * 3 + type] = c;
  }
}

__global__ void csr_rev_count_kernel(const uint32_t* __restrict__ pairs, uint64_t P, int type, uint64_t n,
                                     uint32_t* __restrict__ cnt) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += stride) {
    const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
    if (b < n && a != b) atomicAdd(&cnt[static_cast<uint64_t>(b) * 3 + type], 1u);
  }
}

// The forward entries of point i's segment in pair order, one warp per point (coalesced reads and writes).
__global__ void __launch_bounds__(256) csr_fwd_fill_kernel(const uint32_t* __restrict__ pairs, uint64_t n,
                                                           uint32_t k, int type, const uint32_t* __restrict__ rp,
                                                           uint32_t* __restrict__ col) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31;
  if (i >= n) return;
  uint32_t pos = rp[i * 3 + type];
  for (uint32_t q0 = 0; q0 < k; q0 += 32) {
    const uint32_t q = q0 + lane;
    const uint32_t j = q < k ? pairs[2 * (i * k + q) + 1] : 0xFFFFFFFFu;
    const bool keep = q < k && j < n && j != i;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) col[pos + __popc(bal & ((1u << lane) - 1u))] = j;
    pos += __popc(bal);
  }
}

// Reverse entries: pair (a, b) puts a into b's segment at a cursor taken by atomicAdd. Four pairs per round
// have their atomics in flight together (a thread would otherwise wait one round trip per pair); the
// order inside a segment is the atomics' and is sorted afterwards.
__global__ void csr_rev_fill_kernel(const uint32_t* __restrict__ pairs, uint64_t P, int type, uint64_t n,
                                    uint32_t* __restrict__ cursor, uint32_t* __restrict__ col) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; p + 3 * stride < P; p += 4 * stride) {
    uint32_t a[4], b[4], pos[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      a[k] = pairs[2 * (p + k * stride)];
      b[k] = pairs[2 * (p + k * stride) + 1];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      pos[k] = (b[k] < n && a[k] != b[k]) ? atomicAdd(&cursor[static_cast<uint64_t>(b[k]) * 3 + type], 1u) : 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (b[k] < n && a[k] != b[k]) col[pos[k]] = a[k];
  }
  for (; p < P; p += stride) {
    const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
    if (b < n && a != b) col[atomicAdd(&cursor[static_cast<uint64_t>(b) * 3 + type], 1u)] = a;
  }
}

__global__ void add_offsets_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t len,
                                   uint32_t* __restrict__ out) {
  const uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s < len) out[s] = a[s] + b[s];
}

// Exclusive scan of u32 counts (the host checks that the total fits in u32).
constexpr int SCAN_T = 256, SCAN_PER = 8, SCAN_TILE = SCAN_T * SCAN_PER;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* tmp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) tmp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (SCAN_T / 32) ? tmp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < (SCAN_T / 32)) tmp[lane] = wi - w;
    if (lane == (SCAN_T / 32) - 1) tmp[SCAN_T / 32] = wi;
  }
  __syncthreads();
  const uint32_t res = tmp[warp] + incl - v;
  total = tmp[SCAN_T / 32];
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(SCAN_T) scan_tiles_kernel(const uint32_t* __restrict__ in, uint64_t len,
                                                            uint32_t* __restrict__ out, uint32_t* __restrict__ sums) {
  __shared__ uint32_t tmp[SCAN_T / 32 + 1];
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * SCAN_TILE + threadIdx.x * SCAN_PER;
  uint32_t v[SCAN_PER], s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) {
    v[q] = (base + q < len) ? in[base + q] : 0u;
    s += v[q];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, tmp, total);
#pragma unroll
  for (int q = 0; q < SCAN_PER; ++q) {
    if (base + q < len) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) scan_sums_kernel(uint32_t* __restrict__ sums, uint64_t len) {
  __shared__ uint32_t tmp[SCAN_T / 32 + 1];
  uint32_t carry = 0;
  for (uint64_t b0 = 0; b0 < len; b0 += SCAN_T) {
    const uint64_t i = b0 + threadIdx.x;
    const uint32_t v = i < len ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, tmp, total);
    if (i < len) sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void scan_add_kernel(uint32_t* __restrict__ out, uint64_t len, const uint32_t* __restrict__ sums) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < len) out[i] += sums[i / SCAN_TILE];
}

// Segment sort: one warp per segment of <= 1024 entries in shared memory; longer segments are
// listed for a block-level pass.
constexpr int SEG_WARPS = 8, SEG_SMALL = 1024, SEG_MID = 32768;

template <typename T>
__device__ __forceinline__ void bitonic_sort_range(T* s, int len, int tid, int nthreads, bool block) {
  for (int size = 2; size <= len; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (block) __syncthreads(); else __syncwarp();
      for (int t = tid; t < (len >> 1); t += nthreads) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = ((i & size) == 0);
        const T a = s[i], b = s[j];
        if ((a > b) == up) {
          s[i] = b;
          s[j] = a;
        }
      }
    }
  }
  if (block) __syncthreads(); else __syncwarp();
}

// skip (may be null): the first skip[s] entries of segment s are already in their final order. The
// neighbour segments (type 0) are sorted whole all the same: a point and its neighbour are often each
// other's neighbours, and sorting puts the two entries of such a pair side by side, where the gradient
// kernel's lanes read the partner's coordinates in one request instead of two.
__device__ __forceinline__ uint32_t seg_skip(const uint32_t* __restrict__ skip, uint64_t sidx) {
  return (skip && sidx % 3 != 0) ? skip[sidx] : 0u;
}

__global__ void __launch_bounds__(SEG_WARPS * 32) seg_sort_small_kernel(const uint32_t* __restrict__ rp,
                                                                        const uint32_t* __restrict__ skip,
                                                                        uint32_t* __restrict__ col, uint64_t nseg,
                                                                        uint32_t* __restrict__ big,
                                                                        uint32_t* __restrict__ nbig) {
  __shared__ uint32_t buf[SEG_WARPS][SEG_SMALL];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t sidx = static_cast<uint64_t>(blockIdx.x) * SEG_WARPS + warp; sidx < nseg;
       sidx += static_cast<uint64_t>(gridDim.x) * SEG_WARPS) {
    const uint32_t b = rp[sidx] + seg_skip(skip, sidx), e = rp[sidx + 1];
    const int len = static_cast<int>(e - b);
    if (len <= 1) continue;
    if (len > SEG_SMALL) {
      if (lane == 0) big[atomicAdd(nbig, 1u)] = static_cast<uint32_t>(sidx);
      continue;
    }
    if (len <= 128) {  // in registers: up to 4 keys per lane
      auto sort_regs = [&](auto tag) {
        constexpr int R = decltype(tag)::value;
        uint32_t v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int t = r * 32 + lane;
          v[r] = t < len ? col[b + t] : 0xFFFFFFFFu;
        }
        warp_sort_regs_u32<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int t = r * 32 + lane;
          if (t < len) col[b + t] = v[r];
        }
      };
      if (len <= 32) sort_regs(std::integral_constant<int, 1>());
      else if (len <= 64) sort_regs(std::integral_constant<int, 2>());
      else sort_regs(std::integral_constant<int, 4>());
      continue;
    }
    const int P = next_pow2(len);
    for (int t = lane; t < P; t += 32) buf[warp][t] = t < len ? col[b + t] : 0xFFFFFFFFu;
    bitonic_sort_range<uint32_t>(buf[warp], P, lane, 32, false);
    for (int t = lane; t < len; t += 32) col[b + t] = buf[warp][t];
    __syncwarp();
  }
}

__global__ void __launch_bounds__(1024) seg_sort_mid_kernel(const uint32_t* __restrict__ rp,
                                                            const uint32_t* __restrict__ skip,
                                                            uint32_t* __restrict__ col,
                                                            const uint32_t* __restrict__ big, uint32_t nbig) {
  extern __shared__ uint32_t mbuf[];
  for (uint32_t q = blockIdx.x; q < nbig; q += gridDim.x) {
    const uint32_t sidx = big[q];
    const uint32_t b = rp[sidx] + seg_skip(skip, sidx), e = rp[sidx + 1];
    const int len = static_cast<int>(e - b);
    if (len > SEG_MID) continue;
    const int P = next_pow2(len);
    __syncthreads();
    for (int t = threadIdx.x; t < P; t += blockDim.x) mbuf[t] = t < len ? col[b + t] : 0xFFFFFFFFu;
    bitonic_sort_range<uint32_t>(mbuf, P, threadIdx.x, blockDim.x, true);
    for (int t = threadIdx.x; t < len; t += blockDim.x) col[b + t] = mbuf[t];
  }
}

// Segments beyond shared memory: a bitonic network over a power-of-two global scratch, one block.
__global__ void __launch_bounds__(1024) seg_sort_huge_kernel(uint32_t* __restrict__ col, uint32_t b, uint32_t len,
                                                             uint32_t* __restrict__ scratch, uint32_t P) {
  for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) scratch[t] = t < len ? col[b + t] : 0xFFFFFFFFu;
  bitonic_sort_range<uint32_t>(scratch, static_cast<int>(P), threadIdx.x, blockDim.x, true);
  for (uint32_t t = threadIdx.x; t < len; t += blockDim.x) col[b + t] = scratch[t];
}

// ------------------------------------------------------------------------------------------------
// Initialisation
// ------------------------------------------------------------------------------------------------
constexpr int INIT_MAX_DIM = 16;
constexpr int STD_BLOCKS = 256;

// Per-block partial sums of (v - mean)^2 in f64, one row of partials per block (fixed order).
__global__ void __launch_bounds__(256) var_partial_kernel(const float* __restrict__ v, uint64_t n, int dim,
                                                          const float* __restrict__ mean,
                                                          double* __restrict__ partial) {
  __shared__ double red[256];
  for (int cc = 0; cc < dim; ++cc) {
    double s = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
      const double df = static_cast<double>(v[i * dim + cc]) - static_cast<double>(mean[cc]);
      s += df * df;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[static_cast<uint64_t>(blockIdx.x) * dim + cc] = red[0];
    __syncthreads();
  }
}

__global__ void std_final_kernel(const double* __restrict__ partial, int nblocks, int dim, uint64_t n,
                                 float* __restrict__ sd) {
  const int cc = threadIdx.x;
  if (cc >= dim) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partial[static_cast<uint64_t>(b) * dim + cc];
  sd[cc] = static_cast<float>(sqrt(s / static_cast<double>(n)));
}

__global__ void zscore_kernel(const float* __restrict__ v, uint64_t total, int dim, const float* __restrict__ mean,
                              const float* __restrict__ sd, float* __restrict__ y) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int cc = static_cast<int>(t % dim);
    const float a = __fmul_rn(__fsub_rn(v[t], mean[cc]), 0.0001f);
    y[t] = __fdiv_rn(a, sd[cc]);
  }
}

__global__ void random_init_kernel(uint64_t total, uint64_t seed, float* __restrict__ y) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t q = t >> 1;
    uint32_t w[4];
    philox4x32_10(static_cast<uint32_t>(q), static_cast<uint32_t>(q >> 32), 0u, TAG_INIT, static_cast<uint32_t>(seed),
                  static_cast<uint32_t>(seed >> 32), w);
    const double u1 = (static_cast<double>(w[0] >> 8) + 1.0) * (1.0 / 16777216.0);
    const double u2 = static_cast<double>(w[1] >> 8) * (1.0 / 16777216.0);
    const double r = sqrt(-2.0 * log(u1));
    const double a = 6.283185307179586476925286766559 * u2;
    y[t] = static_cast<float>((t & 1) ? r * sin(a) : r * cos(a));
  }
}

// ------------------------------------------------------------------------------------------------
// K8: fused gradient + Adam
// ------------------------------------------------------------------------------------------------
struct Sched {
  float w_nn, w_mn, w_fp, lr_t;
};

// y of partner j (DIM consecutive floats; one 8-byte load for 2-D).
template <int DIM>
__device__ __forceinline__ void load_y(const float* __restrict__ y, uint32_t j, float (&out)[DIM]) {
  if constexpr (DIM == 2) {
    const float2 v = *reinterpret_cast<const float2*>(y + static_cast<uint64_t>(j) * 2);
    out[0] = v.x;
    out[1] = v.y;
  } else {
#pragma unroll
    for (int c = 0; c < DIM; ++c) out[c] = y[static_cast<uint64_t>(j) * DIM + c];
  }
}

// One segment (one pair type) of a row: lane gl of a G-lane group takes entries s + gl, s + gl + G, ...
// in that order, with the partner index and y of the next entry loaded ahead (two-deep pipeline).
// The type's constants (c1, c2, weight, sign) are fixed for the whole segment.
template <int DIM, bool REPULSIVE>
__device__ __forceinline__ void accumulate_segment(const float* __restrict__ y, const uint32_t* __restrict__ col,
                                                   uint32_t s, uint32_t e, int gl, int G, const float (&yi)[DIM],
                                                   float c1, float c2, float w, float (&acc)[DIM], float& lacc,
                                                   bool want_loss) {
  uint32_t j = s + static_cast<uint32_t>(gl);
  if (j >= e) return;
  const uint32_t g = static_cast<uint32_t>(G);
  uint32_t ja = col[j];
  uint32_t jb = j + g < e ? col[j + g] : 0u;
  float ya[DIM];
  load_y<DIM>(y, ja, ya);
  for (; j < e; j += g) {
    float yb[DIM];
    if (j + g < e) load_y<DIM>(y, jb, yb);
    const uint32_t jc = j + 2 * g < e ? col[j + 2 * g] : 0u;
    float df[DIM];
    float dsq = 1.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      df[c] = __fsub_rn(yi[c], ya[c]);
      dsq = __fadd_rn(dsq, __fmul_rn(df[c], df[c]));
    }
    const float tt = __fadd_rn(c1, dsq);
    const float w1 = __fmul_rn(w, __fdiv_rn(c2, __fmul_rn(tt, tt)));
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const float gterm = __fmul_rn(w1, df[c]);
      acc[c] = __fadd_rn(acc[c], REPULSIVE ? -gterm : gterm);
    }
    if (want_loss)
      lacc += REPULSIVE ? __fmul_rn(w, __fdiv_rn(1.0f, __fadd_rn(1.0f, dsq))) : __fmul_rn(w, __fdiv_rn(dsq, tt));
#pragma unroll
    for (int c = 0; c < DIM; ++c) ya[c] = yb[c];
    jb = jc;
  }
}

// A row's forces: the NN, MN (skipped when w_mn = 0) and FP segments in turn (per-pair arithmetic of
// gradient.rs:120-147: c = 10, 10000 and 1 in the denominators, FP repulsive).
template <int DIM>
__device__ __forceinline__ void accumulate_row(const float* __restrict__ y, const uint32_t* __restrict__ col,
                                               uint32_t s0, uint32_t s1, uint32_t s2, uint32_t s3, bool use_mn,
                                               int gl, int G, const float (&yi)[DIM], const Sched& sc,
                                               float (&acc)[DIM], float& lacc, bool want_loss) {
  accumulate_segment<DIM, false>(y, col, s0, s1, gl, G, yi, 10.0f, 20.0f, sc.w_nn, acc, lacc, want_loss);
  if (use_mn)
    accumulate_segment<DIM, false>(y, col, s1, s2, gl, G, yi, 10000.0f, 20000.0f, sc.w_mn, acc, lacc, want_loss);
  accumulate_segment<DIM, true>(y, col, s2, s3, gl, G, yi, 1.0f, 2.0f, sc.w_fp, acc, lacc, want_loss);
}

template <int G, int DIM>
__global__ void __launch_bounds__(256) grad_adam_kernel(const float* __restrict__ y_cur, float* __restrict__ y_next,
                                                        float* __restrict__ m, float* __restrict__ v,
                                                        const uint32_t* __restrict__ rp,
                                                        const uint32_t* __restrict__ col, uint64_t n,
                                                        const Sched* __restrict__ sched, int itr, float a1, float a2,
                                                        float* __restrict__ row_loss, float* __restrict__ grad_out,
                                                        int grad_only) {
  const Sched sc = sched[itr];
  const int gl = threadIdx.x & (G - 1);
  const uint64_t groups = static_cast<uint64_t>(gridDim.x) * (blockDim.x / G);
  const bool want_loss = row_loss != nullptr;
  const unsigned gmask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / G) + threadIdx.x / G; i < n; i += groups) {
    float yi[DIM], acc[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      yi[c] = y_cur[i * DIM + c];
      acc[c] = 0.0f;
    }
    float lacc = 0.0f;
    const uint32_t s0 = rp[3 * i], s1 = rp[3 * i + 1], s2 = rp[3 * i + 2], s3 = rp[3 * i + 3];
    accumulate_row<DIM>(y_cur, col, s0, s1, s2, s3, sc.w_mn != 0.0f, gl, G, yi, sc, acc, lacc, want_loss);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) acc[c] = __fadd_rn(acc[c], __shfl_xor_sync(gmask, acc[c], o, G));
      if (want_loss) lacc += __shfl_xor_sync(gmask, lacc, o, G);
    }
    if (gl == 0 && grad_only) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) grad_out[i * DIM + c] = acc[c];
      if (want_loss) row_loss[i] = lacc;
    } else if (gl == 0) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float g = acc[c];
        float mm = m[i * DIM + c], vv = v[i * DIM + c];
        mm = __fadd_rn(mm, __fmul_rn(a1, __fsub_rn(g, mm)));
        vv = __fadd_rn(vv, __fmul_rn(a2, __fsub_rn(__fmul_rn(g, g), vv)));
        const float step = __fdiv_rn(__fmul_rn(sc.lr_t, mm), __fadd_rn(__fsqrt_rn(vv), 1e-7f));
        m[i * DIM + c] = mm;
        v[i * DIM + c] = vv;
        y_next[i * DIM + c] = __fsub_rn(yi[c], step);
        if (grad_out) grad_out[i * DIM + c] = g;
      }
      if (want_loss) row_loss[i] = lacc;
    }
  }
}

// Sum of the per-row losses in a fixed order; each pair was counted at both endpoints.
__global__ void __launch_bounds__(1024) loss_reduce_kernel(const float* __restrict__ row_loss, uint64_t n,
                                                           float* __restrict__ out) {
  __shared__ double red[1024];
  double s = 0.0;
  for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) s += row_loss[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = static_cast<float>(0.5 * red[0]);
}

using GradFn = void (*)(const float*, float*, float*, float*, const uint32_t*, const uint32_t*, uint64_t, const Sched*,
                        int, float, float, float*, float*, int);

template <int G>
GradFn pick_grad_kernel(uint64_t dim) {
  switch (dim) {
    case 1: return grad_adam_kernel<G, 1>;
    case 2: return grad_adam_kernel<G, 2>;
    case 3: return grad_adam_kernel<G, 3>;
    case 4: return grad_adam_kernel<G, 4>;
    case 5: return grad_adam_kernel<G, 5>;
    case 6: return grad_adam_kernel<G, 6>;
    case 7: return grad_adam_kernel<G, 7>;
    case 8: return grad_adam_kernel<G, 8>;
    default: return nullptr;
  }
}

// compiler-rt __powisf2 (Rust f32::powi with a run-time exponent).
float powi_f32(float a, int b) {
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

// weights.rs:52-81 and adam.rs:45-47 (file lines) in the reference's f32 arithmetic.
Sched schedule_at(uint64_t itr, uint64_t p1, uint64_t p2, float lr) {
  Sched s;
  if (itr < p1) {
    const float progress = static_cast<float>(itr) / static_cast<float>(p1);
    const float a = (1.0f - progress) * 1000.0f;
    const float b = progress * 3.0f;
    s.w_mn = a + b;
    s.w_nn = 2.0f;
    s.w_fp = 1.0f;
  } else if (itr < p1 + p2) {
    s.w_mn = 3.0f;
    s.w_nn = 3.0f;
    s.w_fp = 1.0f;
  } else {
    s.w_mn = 0.0f;
    s.w_nn = 1.0f;
    s.w_fp = 1.0f;
  }
  const int t = static_cast<int>(itr + 1);
  const float sq = std::sqrt(1.0f - powi_f32(0.999f, t));
  const float q = 1.0f - powi_f32(0.9f, t);
  s.lr_t = (lr * sq) / q;
  return s;
}

}  // namespace

void build_csr(Ctx& c, uint64_t n, const uint32_t* d_pnn, uint64_t n_nn, const uint32_t* d_pmn, uint64_t n_mn,
               const uint32_t* d_pfp, uint64_t n_fp, Csr& out, bool grouped_known) {
  PM_REQUIRE(n < (1ull << 32), PACMAP_ERR_UNSUPPORTED, "pair indices are u32: n must be < 2^32");
  PM_REQUIRE(2 * (n_nn + n_mn + n_fp) < 0xFFFFFFFFull, PACMAP_ERR_UNSUPPORTED, "more than 2^31 pairs");
  const uint64_t nseg = 3 * n;
  DevBuf<uint32_t> cnt(c, nseg + 1);
  PM_CUDA(cudaMemsetAsync(cnt.get(), 0, (nseg + 1) * sizeof(uint32_t), c.stream));
  const uint32_t* lists[3] = {d_pnn, d_pmn, d_pfp};
  const uint64_t sizes[3] = {n_nn, n_mn, n_fp};
  auto grid_for = [&](uint64_t items) {
    return static_cast<unsigned>(std::min<uint64_t>(ceil_div(items, 256), c.sm_count * 16ull));
  };
  // Are the lists grouped by point (every generated list is)? Then forward entries need no atomics.
  bool grouped = n > 0;
  for (int t = 0; t < 3 && grouped; ++t) grouped = sizes[t] % n == 0 && sizes[t] / n < (1ull << 31);
  DevBuf<uint32_t> flag, fwd;
  if (grouped && !grouped_known) {
    flag.alloc(c, 1);
    const uint32_t one = 1u;
    PM_CUDA(cudaMemcpyAsync(flag.get(), &one, sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      grouped_check_kernel<<<grid_for(sizes[t]), 256, 0, c.stream>>>(lists[t], sizes[t],
                                                                     static_cast<uint32_t>(sizes[t] / n), flag.get());
      PM_LAUNCHED();
    }
    uint32_t h = 0;
    PM_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    grouped = h != 0;
  }
  if (grouped) {
    fwd.alloc(c, nseg);
    PM_CUDA(cudaMemsetAsync(fwd.get(), 0, nseg * sizeof(uint32_t), c.stream));
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_fwd_count_kernel<<<ceil_div(n, 8), 256, 0, c.stream>>>(lists[t], n, static_cast<uint32_t>(sizes[t] / n), t,
                                                                fwd.get(), cnt.get(), c.d_err);
      PM_LAUNCHED();
    }
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_rev_count_kernel<<<grid_for(sizes[t]), 256, 0, c.stream>>>(lists[t], sizes[t], t, n, cnt.get());
      PM_LAUNCHED();
    }
  } else {
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_count_kernel<<<grid_for(sizes[t]), 256, 0, c.stream>>>(lists[t], sizes[t], t, n, cnt.get(), c.d_err);
      PM_LAUNCHED();
    }
  }
  c.check_errors("pair lists");
  out.row_ptr.alloc(c, nseg + 1);
  const uint64_t tiles = ceil_div(nseg + 1, SCAN_TILE);
  DevBuf<uint32_t> sums(c, tiles);
  scan_tiles_kernel<<<static_cast<unsigned>(tiles), SCAN_T, 0, c.stream>>>(cnt.get(), nseg + 1, out.row_ptr.get(),
                                                                          sums.get());
  PM_LAUNCHED();
  scan_sums_kernel<<<1, SCAN_T, 0, c.stream>>>(sums.get(), tiles);
  PM_LAUNCHED();
  scan_add_kernel<<<ceil_div(nseg + 1, 256), 256, 0, c.stream>>>(out.row_ptr.get(), nseg + 1, sums.get());
  PM_LAUNCHED();
  uint32_t total = 0;
  PM_CUDA(cudaMemcpyAsync(&total, out.row_ptr.get() + nseg, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  out.entries = total;
  out.col.alloc(c, std::max<uint64_t>(total, 1));
  if (grouped) {
    // forward entries in pair order; reverse entries after them by atomics (cursor = row_ptr + forward)
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_fwd_fill_kernel<<<ceil_div(n, 8), 256, 0, c.stream>>>(lists[t], n, static_cast<uint32_t>(sizes[t] / n), t,
                                                               out.row_ptr.get(), out.col.get());
      PM_LAUNCHED();
    }
    add_offsets_kernel<<<ceil_div(nseg, 256), 256, 0, c.stream>>>(out.row_ptr.get(), fwd.get(), nseg, cnt.get());
    PM_LAUNCHED();
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_rev_fill_kernel<<<grid_for(sizes[t]), 256, 0, c.stream>>>(lists[t], sizes[t], t, n, cnt.get(),
                                                                    out.col.get());
      PM_LAUNCHED();
    }
  } else {
    // cursor = row_ptr (reuse the count buffer)
    PM_CUDA(cudaMemcpyAsync(cnt.get(), out.row_ptr.get(), (nseg + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            c.stream));
    for (int t = 0; t < 3; ++t) {
      if (!sizes[t]) continue;
      csr_fill_kernel<<<grid_for(sizes[t]), 256, 0, c.stream>>>(lists[t], sizes[t], t, n, cnt.get(), out.col.get());
      PM_LAUNCHED();
    }
  }
  // sort what the atomics placed: whole segments, or (grouped) the reverse part after the forward entries
  const uint32_t* skip = grouped ? fwd.get() : nullptr;
  DevBuf<uint32_t> big(c, nseg + 1);
  PM_CUDA(cudaMemsetAsync(big.get() + nseg, 0, sizeof(uint32_t), c.stream));
  const unsigned g = static_cast<unsigned>(std::min<uint64_t>(ceil_div(nseg, SEG_WARPS), c.sm_count * 8ull));
  seg_sort_small_kernel<<<g, SEG_WARPS * 32, 0, c.stream>>>(out.row_ptr.get(), skip, out.col.get(), nseg, big.get(),
                                                           big.get() + nseg);
  PM_LAUNCHED();
  uint32_t nbig = 0;
  PM_CUDA(cudaMemcpyAsync(&nbig, big.get() + nseg, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  if (nbig > 0) {
    const size_t smem = SEG_MID * sizeof(uint32_t);
    PM_CUDA(cudaFuncSetAttribute(seg_sort_mid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    seg_sort_mid_kernel<<<std::min<uint32_t>(nbig, c.sm_count * 2), 1024, smem, c.stream>>>(
        out.row_ptr.get(), skip, out.col.get(), big.get(), nbig);
    PM_LAUNCHED();
    // Segments longer than shared memory (points that appear in > 32768 pairs of one type).
    std::vector<uint32_t> hb(nbig), hrp(nseg + 1), hskip;
    PM_CUDA(cudaMemcpyAsync(hb.data(), big.get(), nbig * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(hrp.data(), out.row_ptr.get(), (nseg + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            c.stream));
    if (skip) {
      hskip.resize(nseg);
      PM_CUDA(cudaMemcpyAsync(hskip.data(), skip, nseg * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
    }
    PM_CUDA(cudaStreamSynchronize(c.stream));
    DevBuf<uint32_t> scratch;
    for (uint32_t q = 0; q < nbig; ++q) {
      const uint32_t b = hrp[hb[q]] + ((skip && hb[q] % 3 != 0) ? hskip[hb[q]] : 0u), len = hrp[hb[q] + 1] - b;
      if (len <= static_cast<uint32_t>(SEG_MID)) continue;
      const uint32_t P = static_cast<uint32_t>(next_pow2(static_cast<int>(len)));
      if (scratch.count < P) scratch.alloc(c, P);
      seg_sort_huge_kernel<<<1, 1024, 0, c.stream>>>(out.col.get(), b, len, scratch.get(), P);
      PM_LAUNCHED();
    }
  }
}

void init_value_device(Ctx& c, const float* d_v, uint64_t n, uint64_t dim, float* d_y) {
  PM_REQUIRE(n > 0, PACMAP_ERR_EMPTY_ARRAY_MEAN, "Failed to calculate mean axis: the array is empty");
  PM_REQUIRE(dim <= INIT_MAX_DIM, PACMAP_ERR_UNSUPPORTED, "embedding dimensions above 16 are not supported");
  if (dim == 0) return;
  DevBuf<float> mean(c, dim), sd(c, dim);
  DevBuf<double> partial(c, static_cast<size_t>(STD_BLOCKS) * dim);
  column_mean_seq(c, d_v, n, dim, 0.0f, 1.0f, mean.get());
  var_partial_kernel<<<STD_BLOCKS, 256, 0, c.stream>>>(d_v, n, static_cast<int>(dim), mean.get(), partial.get());
  PM_LAUNCHED();
  std_final_kernel<<<1, 32, 0, c.stream>>>(partial.get(), STD_BLOCKS, static_cast<int>(dim), n, sd.get());
  PM_LAUNCHED();
  const uint64_t total = n * dim;
  zscore_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), c.sm_count * 16ull)), 256, 0,
                  c.stream>>>(d_v, total, static_cast<int>(dim), mean.get(), sd.get(), d_y);
  PM_LAUNCHED();
}

void init_random_device(Ctx& c, uint64_t n, uint64_t dim, uint64_t seed, float* d_y) {
  const uint64_t total = n * dim;
  if (!total) return;
  random_init_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), c.sm_count * 16ull)), 256, 0,
                       c.stream>>>(total, seed, d_y);
  PM_LAUNCHED();
}

double& last_graph_setup_ms() {
  static thread_local double v = 0.0;
  return v;
}

void optimize_device(Ctx& c, const Csr& csr, const OptimizeArgs& a) {
  const uint64_t n = a.n, dim = a.dim;
  if (a.itr_end <= a.itr_begin || n == 0 || dim == 0) return;
  PM_REQUIRE(dim <= 8, PACMAP_ERR_UNSUPPORTED, "the optimiser supports embedding dimensions 1..8");
  constexpr int G = 8;
  GradFn fn = pick_grad_kernel<G>(dim);
  const uint64_t total_iters = a.p1 + a.p2 + a.p3;
  const uint64_t sched_len = std::max<uint64_t>(total_iters, a.itr_end);
  std::vector<Sched> hs(sched_len);
  for (uint64_t t = 0; t < sched_len; ++t) hs[t] = schedule_at(t, a.p1, a.p2, a.lr);
  DevBuf<Sched> sched(c, sched_len);
  PM_CUDA(cudaMemcpyAsync(sched.get(), hs.data(), sched_len * sizeof(Sched), cudaMemcpyHostToDevice, c.stream));
  const float a1 = 1.0f - 0.9f, a2 = 1.0f - 0.999f;

  DevBuf<float> yb(c, n * dim);
  DevBuf<float> row_loss, loss_dev;
  const uint64_t iters = a.itr_end - a.itr_begin;
  if (a.h_loss) {
    row_loss.alloc(c, n);
    loss_dev.alloc(c, iters);
  }
  int per_sm = 0;
  PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0));
  const unsigned grid = static_cast<unsigned>(
      std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, 256 / G), static_cast<uint64_t>(c.sm_count) * std::max(per_sm, 1))));
  float* bufs[2] = {a.d_y, yb.get()};

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const auto setup_t0 = std::chrono::steady_clock::now();
  PM_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
  uint64_t launches = 0;
  bool capture_ok = true;
  std::string capture_msg;
  for (uint64_t itr = a.itr_begin; itr < a.itr_end; ++itr) {
    const int src = static_cast<int>((itr - a.itr_begin) & 1), dst = src ^ 1;
    fn<<<grid, 256, 0, c.stream>>>(bufs[src], bufs[dst], a.d_m, a.d_v, csr.row_ptr.get(), csr.col.get(), n,
                                   sched.get(), static_cast<int>(itr), a1, a2, a.h_loss ? row_loss.get() : nullptr,
                                   (itr + 1 == a.itr_end) ? a.d_grad_last : nullptr, 0);
    ++launches;
    if (a.h_loss) {
      loss_reduce_kernel<<<1, 1024, 0, c.stream>>>(row_loss.get(), n, loss_dev.get() + (itr - a.itr_begin));
      ++launches;
    }
    if (a.d_snap && a.snapshots) {
      for (uint64_t sidx = 0; sidx < a.n_snapshots; ++sidx) {
        if (a.snapshots[sidx] == itr + 1) {
          if (cudaMemcpyAsync(a.d_snap + sidx * n * dim, bufs[dst], n * dim * sizeof(float), cudaMemcpyDeviceToDevice,
                              c.stream) != cudaSuccess) {
            capture_ok = false;
            capture_msg = "snapshot copy";
          }
          break;
        }
      }
    }
  }
  const cudaError_t end_err = cudaStreamEndCapture(c.stream, &graph);
  if (!capture_ok || end_err != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    throw Fail{PACMAP_ERR_CUDA, "graph capture failed: " + capture_msg + " " + cudaGetErrorString(end_err)};
  }
  const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
  last_graph_setup_ms() =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - setup_t0).count();
  if (inst != cudaSuccess) {
    cudaGraphDestroy(graph);
    throw Fail{PACMAP_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(inst)};
  }
  const cudaError_t lerr = cudaGraphLaunch(exec, c.stream);
  count_launch(launches);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  PM_CUDA(lerr);
  if ((iters & 1) == 1)
    PM_CUDA(cudaMemcpyAsync(a.d_y, yb.get(), n * dim * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
  if (a.h_loss) {
    PM_CUDA(cudaMemcpyAsync(a.h_loss, loss_dev.get(), iters * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  }
  PM_CUDA(cudaStreamSynchronize(c.stream));
}

void gradient_device(Ctx& c, const Csr& csr, const float* d_y, uint64_t n, uint64_t dim, float w_nn, float w_mn,
                     float w_fp, float* d_grad, float* h_loss) {
  if (n == 0 || dim == 0) return;
  PM_REQUIRE(dim <= 8, PACMAP_ERR_UNSUPPORTED, "the optimiser supports embedding dimensions 1..8");
  constexpr int G = 8;
  GradFn fn = pick_grad_kernel<G>(dim);
  const Sched hs{w_nn, w_mn, w_fp, 0.0f};
  DevBuf<Sched> sched(c, 1);
  DevBuf<float> row_loss(c, n), loss_dev(c, 1);
  PM_CUDA(cudaMemcpyAsync(sched.get(), &hs, sizeof(Sched), cudaMemcpyHostToDevice, c.stream));
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n, 256 / G), c.sm_count * 8ull));
  fn<<<grid, 256, 0, c.stream>>>(d_y, nullptr, nullptr, nullptr, csr.row_ptr.get(), csr.col.get(), n, sched.get(), 0,
                                 0.0f, 0.0f, row_loss.get(), d_grad, 1);
  PM_LAUNCHED();
  loss_reduce_kernel<<<1, 1024, 0, c.stream>>>(row_loss.get(), n, loss_dev.get());
  PM_LAUNCHED();
  PM_CUDA(cudaMemcpyAsync(h_loss, loss_dev.get(), sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace pacmap
