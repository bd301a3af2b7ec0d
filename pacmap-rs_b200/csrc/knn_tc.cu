// Exact kNN through a tensor-core filter (tcgen05 + TMA + TMEM) and an exact FP32 re-rank.
//
// The reference ranks neighbours by its f32 distance (src/knn.rs:149-191, src/distance.rs:50-75). Here
// the O(n^2 d) part runs as a distance GEMM on the 5th-generation tensor cores and only a small,
// provably complete candidate set per row is re-ranked with the reference's exact f32 arithmetic:
//
//  1. prep: x is scaled by an exact power of two s (max |x s| < 2^13), split into h = fp16(x s) (or
//     bf16) and l = x s - h; per point n = ||x s||^2, A = ||h||^2, B = ||l||^2 (f32).
//  2. knn_filter_kernel: per 256-row block, G = h_i . h_j for every column tile of 128 points by
//     tcgen05.mma (M=128 x2 halves, N=128, K=16 steps, FP32 accumulators in TMEM, operands staged by
//     TMA with 128-byte swizzle). The epilogue forms v_ij = (n_j - 2 e_j) - 2 G_ij.
//     Error bound: with e_j = (rho A_j + B_j / rho)/2 + B_j/2 + eta A_j/2 + gamma n_j (AM-GM on the
//     Cauchy-Schwarz bound of h.l + l.h + l.l, eta = tensor-core accumulation, gamma = every f32
//     rounding incl. the reference's own distance sum), the reference's squared distance lies in
//     [LB, UB] = [v + n_i - 2e_i, v + 4e_j + n_i + 2e_i].
//     Each row keeps a buffer of candidates (j, v) with v <= theta_i, where theta_i comes from the
//     (k'+1)-th smallest UB seen so far (the +1 covers the row itself); when the buffer fills, the owning
//     warp compacts it (the rank-th smallest by bisection on warp-wide counts; inside the filter the UB of
//     an entry is bounded with the largest e, so no per-entry gather is needed, unless the band would not
//     fit: then again with every entry's own e_j). The final compaction uses every entry's own e_j.
//     Any true neighbour has LB <= k'-th UB, so it is never dropped. From 32,768 rows the tile pruning
//     (knn_prune.cu) restricts each row block to the column tiles that may hold one of its neighbours.
//  3. knn_rerank_kernel: the final threshold, then the reference's exact f32 distance of every
//     survivor (gathered from a lane-grouped copy of x by 16-byte loads, each lane adding its terms in
//     the reference's order), sorted by (distance, index): the rows of knn.rs.
//  Rows whose candidate band does not fit the buffer (e.g. thousands of exact duplicates) are
//  recomputed by the exact SIMT kernel.
//
// Every mbarrier wait is bounded (2 s of %globaltimer): a kernel that gives up raises DEV_ERR_TIMEOUT
// and returns after releasing its tensor memory. No TMA multicast is used anywhere.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "knn_layout.cuh"
#include "knn_prune.cuh"
#include "knn_tc.cuh"
#include "ptx.cuh"
#include "tcgen05.cuh"

namespace pacmap {

namespace {

constexpr int TC_MAX_STAGES = 8;   // operand pipeline depth limit (mbarrier slots)
constexpr int TC_THREADS = 320;    // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2..9 epilogue
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_TMEM_COLS = 512;  // 2 accumulator stages x 2 halves x 128 columns
constexpr int KB_BYTES = 128 * 128;  // one 128-row x 64-element (128 B) swizzled K block
constexpr int G_BYTES = 128 * 32;    // one 128-row x 16-element (32 B) column-term tile

struct alignas(8) TcShared {
  uint64_t full[TC_MAX_STAGES];
  uint64_t empty[TC_MAX_STAGES];
  uint64_t a_full;
  uint64_t tmem_full[2];
  uint64_t tmem_empty[2];
  uint64_t mma_done;
  uint32_t tmem_base;
  int abort_flag;
};

// Operand staging of the filter by data width (KB = K blocks of 64 elements):
//  MODE_TILE   (KB <= 2): the block's A rows stay in shared memory; one stage = every K block of a
//              column tile.
//  MODE_KBLOCK (KB 3..4): A stays resident; one stage = one K block of a column tile.
//  MODE_STREAM (KB >= 5): A no longer fits; one stage = one K block of both A halves and of the column
//              tile (A is re-read from L2 for every tile). KB is a run-time value here.
// The column-term tile rides with the first stage of each column tile.
enum FilterMode { MODE_TILE = 0, MODE_KBLOCK = 1, MODE_STREAM = 2 };
constexpr uint64_t PRUNE_MIN_ROWS = 32768;  // tile pruning from 256 column tiles on
constexpr int PRUNE_PROBE = 2;              // the bound pass: own cells (+ the nearest cell of a small one)
constexpr int TC_SMEM_LIMIT = 232448;  // 227 KB of dynamic shared memory per block
constexpr int FILTER_SLACK = 8;        // the filter's compactions settle for a key within rank + 8 entries
template <int KB, int MODE>
struct FilterLayout {
  static constexpr int A_RES = MODE == MODE_STREAM ? 0 : 2 * KB * KB_BYTES;
  static constexpr int STAGE = (MODE == MODE_TILE ? KB : 1) * KB_BYTES + (MODE == MODE_STREAM ? 2 * KB_BYTES : 0);
  static constexpr int FIT = (TC_SMEM_LIMIT - 1024 - A_RES - G_BYTES - 256) / (STAGE + G_BYTES);
  static constexpr int NST = MODE == MODE_TILE ? 4 : (FIT > TC_MAX_STAGES ? TC_MAX_STAGES : FIT);
  static constexpr size_t SMEM = 1024 + A_RES + static_cast<size_t>(NST + 1) * G_BYTES +
                                 static_cast<size_t>(NST) * STAGE + sizeof(TcShared);
  static_assert(NST >= 2 && SMEM <= TC_SMEM_LIMIT, "filter operands do not fit in shared memory");
};

// ---------------------------------------------------------------------------------------------
// PTX wrappers (sm_100a).
// ---------------------------------------------------------------------------------------------
// ---------------------------------------------------------------------------------------------
// Per-row candidate buffer maintenance (shared by the filter's compaction and the re-rank).
// ---------------------------------------------------------------------------------------------

// theta for row constants (n_i, e4_i = 4 e_i) and the selected u (UB less n_i + 2 e_i): v <= theta keeps
// every candidate whose lower bound is within the (sqrt-tie-widened) k'-th upper bound. Non-decreasing in
// uT, so any uT at or above the rank-th smallest u gives a valid (looser) theta.
__device__ __forceinline__ float theta_from(float uT, float n_i, float e4_i) {
  const float base = uT + e4_i;
  const float slack = 9.5367431640625e-07f * fabsf(uT + n_i + 0.5f * e4_i) + 2.384185791015625e-07f * (n_i + fabsf(uT));
  return base + slack;
}

// Candidate entries are (index j, v = -2 D): v + n_i - 2 e_i is the lower bound of the reference's squared
// distance and u = fl(v + 4 e_j) + n_i + 2 e_i the upper one (scaled by s^2). v is exact (D scaled by -2),
// so the insertion needs no per-column constant and every later u is the same f32 value.
//
// A row's buffer in registers (m <= 32 * PER entries), loaded once per compaction by the whole warp.
template <int PER>
struct RowRegs {
  uint32_t ri[PER];
  float rv[PER];
};
template <int PER>
__device__ __forceinline__ void load_row(const uint2* __restrict__ cand, int m, RowRegs<PER>& r) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = q * 32 + lane;
    const uint2 cv = e < m ? cand[e] : make_uint2(0u, 0u);
    r.ri[q] = cv.x;
    r.rv[q] = __uint_as_float(cv.y);
  }
}

// Compaction of one row's buffer from its registers, one warp: the rank-`rank` smallest u by bisection on
// warp-wide counts, theta from it, and the row's band (v <= theta) written back in order. With ge (the
// separate compaction kernel, and the filter's second compaction) u_j = fl(v_j + 4 e_j) with each entry's
// own e_j. Without it (inside the filter, where a gather per entry would stall the epilogue) the keys are v
// and the rank-th smallest u is bounded by fl(vT + e4max) for the rank-th smallest v = vT (rounding is
// monotone and e4_j <= e4max), a looser but valid theta. theta is capped by theta_cap, an earlier valid
// threshold of the same row (every theta is at or above the row's final one, so the band keeps every
// neighbour; the entries that defined the smaller of the two all pass it, so at least `rank` are kept).
// slack > 0 ends the bisection at the first key T with rank <= #{keys <= T} <= rank + slack: T is then at or
// above the rank-th smallest key (a looser bound, and a band a few entries larger, for fewer serial steps).
template <int PER>
__device__ __forceinline__ int compact_row(uint2* __restrict__ cand, int m, int rank, float n_i, float e4_i,
                                           const RowRegs<PER>& r, float e4max, const float2* __restrict__ ge,
                                           float theta_cap, float& theta_out, uint32_t* ukey_out = nullptr,
                                           int slack = 0) {
  const int lane = threadIdx.x & 31;
  uint32_t rk[PER];
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0u;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const bool in = q * 32 + lane < m;
    float key = r.rv[q];
    if (ge) key = __fadd_rn(key, in ? __ldg(&ge[r.ri[q]].y) : 0.0f);
    rk[q] = in ? total_key(key) : 0xFFFFFFFFu;
    if (in) {
      kmin = min(kmin, rk[q]);
      kmax = max(kmax, rk[q]);
    }
  }
  // The rank-th smallest key by bisection on [min key, max key] with warp-wide counts (no shared
  // memory, no atomics): the smallest key value T with #{keys <= T} >= rank. #{keys <= hi} >= rank holds
  // throughout, so stopping early (slack) leaves hi a valid threshold key.
  uint32_t lo = __reduce_min_sync(0xFFFFFFFFu, kmin), hi = __reduce_max_sync(0xFFFFFFFFu, kmax);
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) cnt += (rk[q] <= mid) ? 1u : 0u;
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    if (cnt >= static_cast<uint32_t>(rank)) {
      hi = mid;
      if (cnt <= static_cast<uint32_t>(rank + slack) && slack > 0) break;
    } else {
      lo = mid + 1u;
    }
  }
  const uint32_t prefix = hi;
  const float uT = ge ? key_to_float(prefix) : __fadd_rn(key_to_float(prefix), e4max);
  const float th = fminf(theta_from(uT, n_i, e4_i), theta_cap);
  int out = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const bool keep = q * 32 + lane < m && r.rv[q] <= th;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) {
      const int pos = out + __popc(bal & ((1u << lane) - 1u));
      cand[pos] = make_uint2(r.ri[q], __float_as_uint(r.rv[q]));
    }
    out += __popc(bal);
  }
  __syncwarp();
  theta_out = th;
  if (ukey_out) *ukey_out = prefix;
  return out;
}

// The band of a buffer that the gather-free compaction left too full, compacted again with every entry's
// own e_j (a tighter theta). Kept out of line: it runs only on hard rows, and the filter's hot loop stays
// small.
template <int PER>
__device__ __noinline__ int recompact_exact(uint2* __restrict__ cand, int m, int rank, float n_i, float e4_i,
                                            const float2* __restrict__ ge, float theta_cap, float& theta_out) {
  RowRegs<PER> r;
  load_row<PER>(cand, m, r);
  return compact_row<PER>(cand, m, min(rank, m), n_i, e4_i, r, 0.0f, ge, theta_cap, theta_out, nullptr,
                          FILTER_SLACK);
}

// ---------------------------------------------------------------------------------------------
// 0. locality order: every point joins the nearest of P pivots (points p * n / P); sorting by pivot
//    puts near points in near rows, so each row block meets its own neighbourhood first (sweep
//    order below) and its threshold tightens after a few tiles. Any order gives the same exact kNN.
// ---------------------------------------------------------------------------------------------
// Register-tiled: a block takes 64 points and the pivots in two passes of 128; each thread keeps 4
// points x 8 pivots of dot products while d is staged through shared memory in slices of 32. Any
// assignment order gives the same kNN; this one only has to be fast. With `score` (n x PIV) it also
// stores |p|^2 - 2 x.p of every (point, pivot) pair, and block 0 stores |p|^2 in `pnorm` (the tile
// pruning's pivot distances).
constexpr int PA_PTS = 64, PA_PIV = 128, PA_D = 32;
constexpr int PA_XS = PA_PTS + 1;  // odd row stride: the transposed writes of x fall in 32 different banks

// The pivots transposed, pT[c * PIV + p] = x[piv_rows[p]][c], zero for d <= c < dpad (dpad = d rounded up to
// PA_D): every block of the assignment then stages its pivot slices with plain 16-byte copies.
__global__ void pivots_t_kernel(const float* __restrict__ x, const uint32_t* __restrict__ piv_rows, int d, int dpad,
                                float* __restrict__ pT) {
  const uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<uint64_t>(dpad) * PIV) return;
  const int c = static_cast<int>(e / PIV), p = static_cast<int>(e % PIV);
  pT[e] = c < d ? x[static_cast<uint64_t>(piv_rows[p]) * d + c] : 0.0f;
}

__global__ void __launch_bounds__(256) pivot_assign_kernel(const float* __restrict__ x, uint64_t n, int d,
                                                           const float* __restrict__ pT,
                                                           uint32_t* __restrict__ cell, float* __restrict__ score,
                                                           float* __restrict__ pnorm) {
  __shared__ float xs[PA_D * PA_XS];                // [dim][point]
  __shared__ __align__(16) float ps[PA_D][PA_PIV];  // [dim][pivot]
  __shared__ float pn[PA_PIV];
  __shared__ float best_s[PA_PTS][16];
  __shared__ uint32_t best_i[PA_PTS][16];
  const uint64_t pt0 = static_cast<uint64_t>(blockIdx.x) * PA_PTS;
  const int tp = threadIdx.x >> 4;  // 16 point groups of 4 points
  const int tq = threadIdx.x & 15;  // 16 pivot groups of 8 pivots
  float best = __int_as_float(0x7f800000);
  uint32_t arg = 0;
  for (int half = 0; half < PIV / PA_PIV; ++half) {
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    float nrm = 0.0f;  // thread t < 128: |pivot t|^2 of this half
    for (int c0 = 0; c0 < d; c0 += PA_D) {
      __syncthreads();
      for (int e = threadIdx.x; e < PA_D * PA_PTS; e += 256) {
        const int pi = e / PA_D, cc = e % PA_D;
        const uint64_t r = pt0 + pi;
        xs[cc * PA_XS + pi] = (r < n && c0 + cc < d) ? x[r * d + c0 + cc] : 0.0f;
      }
      for (int e = threadIdx.x; e < PA_D * PA_PIV / 4; e += 256) {
        const int cc = e / (PA_PIV / 4), v = e % (PA_PIV / 4);
        reinterpret_cast<float4*>(&ps[cc][0])[v] =
            __ldg(reinterpret_cast<const float4*>(pT + static_cast<uint64_t>(c0 + cc) * PIV + half * PA_PIV) + v);
      }
      __syncthreads();
      if (threadIdx.x < PA_PIV)
        for (int cc = 0; cc < PA_D; ++cc) nrm = fmaf(ps[cc][threadIdx.x], ps[cc][threadIdx.x], nrm);
#pragma unroll 8
      for (int cc = 0; cc < PA_D; ++cc) {
        float xv[4], pv[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) xv[i] = xs[cc * PA_XS + tp * 4 + i];
#pragma unroll
        for (int j = 0; j < 8; ++j) pv[j] = ps[cc][tq * 8 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(xv[i], pv[j], acc[i][j]);
      }
    }
    __syncthreads();
    if (threadIdx.x < PA_PIV) {
      pn[threadIdx.x] = nrm;
      if (pnorm && blockIdx.x == 0) pnorm[half * PA_PIV + threadIdx.x] = nrm;
    }
    __syncthreads();
    // per point: the best of this thread's 8 pivots, then of the 16 threads sharing the point
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float b = __int_as_float(0x7f800000);
      uint32_t bi = 0;
      float sc8[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float sc = fmaf(-2.0f, acc[i][j], pn[tq * 8 + j]);
        sc8[j] = sc;
        if (sc < b) {
          b = sc;
          bi = static_cast<uint32_t>(half * PA_PIV + tq * 8 + j);
        }
      }
      const uint64_t pt = pt0 + tp * 4 + i;
      if (score && pt < n) {
        float4* dst = reinterpret_cast<float4*>(score + pt * PIV + half * PA_PIV + tq * 8);
        dst[0] = make_float4(sc8[0], sc8[1], sc8[2], sc8[3]);
        dst[1] = make_float4(sc8[4], sc8[5], sc8[6], sc8[7]);
      }
      best_s[tp * 4 + i][tq] = b;
      best_i[tp * 4 + i][tq] = bi;
    }
    __syncthreads();
    if (threadIdx.x < PA_PTS) {
      for (int q = 0; q < 16; ++q) {
        const float sc = best_s[threadIdx.x][q];
        if (sc < best) {  // ascending pivot order: ties keep the lower pivot
          best = sc;
          arg = best_i[threadIdx.x][q];
        }
      }
    }
  }
  if (threadIdx.x < PA_PTS) {
    const uint64_t i = pt0 + threadIdx.x;
    if (i < n) cell[i] = arg;
  }
}

// The points sorted by cell, stably (ascending index within a cell), so that the order -- and with it the
// row blocks a kNN shard owns -- is the same on every call: per-chunk cell counts, their offsets in
// (cell, chunk) order, then one warp per chunk placing its points in index order.
constexpr uint32_t PL_CHUNK = 4096;
__global__ void __launch_bounds__(256) cell_chunk_count_kernel(const uint32_t* __restrict__ cell, uint64_t n,
                                                               uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[PIV];
  for (int t = threadIdx.x; t < PIV; t += blockDim.x) h[t] = 0;
  __syncthreads();
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * PL_CHUNK, c1 = c0 + PL_CHUNK < n ? c0 + PL_CHUNK : n;
  for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) atomicAdd(&h[cell[i]], 1u);  // a count: any order
  __syncthreads();
  for (int t = threadIdx.x; t < PIV; t += blockDim.x) counts[static_cast<uint64_t>(blockIdx.x) * PIV + t] = h[t];
}

__global__ void __launch_bounds__(PIV) cell_chunk_offsets_kernel(uint32_t* __restrict__ counts, uint32_t chunks) {
  __shared__ uint32_t start[PIV];
  const int t = threadIdx.x;  // one thread per cell
  uint32_t total = 0;
  for (uint32_t ch = 0; ch < chunks; ++ch) total += counts[static_cast<uint64_t>(ch) * PIV + t];
  start[t] = total;
  __syncthreads();
  if (t == 0) {
    uint32_t run = 0;
    for (int p = 0; p < PIV; ++p) {
      const uint32_t v = start[p];
      start[p] = run;
      run += v;
    }
  }
  __syncthreads();
  uint32_t run = start[t];
  for (uint32_t ch = 0; ch < chunks; ++ch) {
    const uint32_t v = counts[static_cast<uint64_t>(ch) * PIV + t];
    counts[static_cast<uint64_t>(ch) * PIV + t] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(32) cell_place_kernel(const uint32_t* __restrict__ cell, uint64_t n,
                                                        const uint32_t* __restrict__ offsets,
                                                        uint32_t* __restrict__ perm) {
  __shared__ uint32_t off[PIV];
  const int lane = threadIdx.x;
  for (int t = lane; t < PIV; t += 32) off[t] = offsets[static_cast<uint64_t>(blockIdx.x) * PIV + t];
  __syncwarp();
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * PL_CHUNK, c1 = c0 + PL_CHUNK < n ? c0 + PL_CHUNK : n;
  for (uint64_t base = c0; base < c1; base += 32) {
    const uint64_t i = base + lane;
    const bool valid = i < c1;
    const uint32_t cl = valid ? cell[i] : 0xFFFFFFFFu;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, cl);
    const int rank = __popc(same & ((1u << lane) - 1u));
    if (valid) perm[off[cl] + rank] = static_cast<uint32_t>(i);
    __syncwarp();
    if (valid && lane == __ffs(same) - 1) off[cl] += __popc(same);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// 1. prep
// ---------------------------------------------------------------------------------------------
__global__ void absmax_kernel(const float* __restrict__ x, uint64_t total, uint32_t* __restrict__ out) {
  uint32_t m = 0;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const float a = fabsf(x[t]);
    if (a == a) m = max(m, __float_as_uint(a));  // NaN excluded
  }
  m = __reduce_max_sync(0xFFFFFFFFu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// The re-rank copy of x: rows in the locality order, each in the lane-grouped layout of the reference's
// eight-lane distance sum (distance.rs:50-75, lane l adds elements l, l + 8, l + 16, ... in turn): lane l's
// terms 4k .. 4k+3 (elements 8 (4k + q) + l) sit at floats 32 k + 4 l + q, zeros past the last full chunk
// of 8, then the d % 8 remainder in order, the row padded to a multiple of 4 floats. An 8-lane group
// reads one 128-byte run per 16-byte load, and each lane still adds its own terms in the reference's
// order (an added zero term leaves an f32 sum unchanged).
struct RerankLayout {
  int nc, nq, tail, ds;  // chunks of 8, groups of 4 chunks, remainder, row stride (floats)
};
__host__ __device__ __forceinline__ RerankLayout rerank_layout(int d) {
  RerankLayout L;
  L.nc = d / 8;
  L.nq = (L.nc + 3) / 4;
  L.tail = d % 8;
  L.ds = 32 * L.nq + ((L.tail + 3) & ~3);
  return L;
}
// The element of x stored at float o of a row in this layout, -1 for padding.
__device__ __forceinline__ int rerank_src(const RerankLayout& L, int o) {
  if (o < 32 * L.nq) {
    const int k = o >> 5, l = (o & 31) >> 2, q = o & 3, p = 4 * k + q;
    return p < L.nc ? 8 * p + l : -1;
  }
  const int t = o - 32 * L.nq;
  return t < L.tail ? 8 * L.nc + t : -1;
}

// Also writes xperm (n rows in the locality order, RerankLayout), which the exact re-rank gathers from.
template <bool BF16>
__global__ void split_rows_kernel(const float* __restrict__ x, const uint32_t* __restrict__ perm, uint64_t n, int d,
                                  int KP, uint64_t n_pad, float s, uint16_t* __restrict__ H, float* __restrict__ nrm,
                                  float* __restrict__ A, float* __restrict__ B, double* __restrict__ partial,
                                  float* __restrict__ xperm) {
  __shared__ double red[2][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double sa = 0.0, sb = 0.0;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * 8 + warp; r < n_pad; r += static_cast<uint64_t>(gridDim.x) * 8) {
    float nn = 0.0f, aa = 0.0f, bb = 0.0f;
    const uint64_t src = r < n ? static_cast<uint64_t>(perm[r]) : 0;
    for (int c = lane; c < KP; c += 32) {
      float xs = 0.0f;
      if (r < n && c < d) {
        const float xv = x[src * d + c];
        xs = xv * s;
      }
      uint16_t hbits;
      float hf;
      if (BF16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(xs);
        hbits = __bfloat16_as_ushort(h);
        hf = __bfloat162float(h);
      } else {
        const __half h = __float2half_rn(xs);
        hbits = __half_as_ushort(h);
        hf = __half2float(h);
      }
      const float l = xs - hf;
      H[r * KP + c] = hbits;
      nn = fmaf(xs, xs, nn);
      aa = fmaf(hf, hf, aa);
      bb = fmaf(l, l, bb);
    }
    if (r < n) {
      const RerankLayout L = rerank_layout(d);
      for (int o = lane; o < L.ds; o += 32) {
        const int c = rerank_src(L, o);
        xperm[r * L.ds + o] = c >= 0 ? x[src * d + c] : 0.0f;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      nn += __shfl_xor_sync(0xFFFFFFFFu, nn, o);
      aa += __shfl_xor_sync(0xFFFFFFFFu, aa, o);
      bb += __shfl_xor_sync(0xFFFFFFFFu, bb, o);
    }
    if (lane == 0 && r < n) {
      nrm[r] = nn;
      A[r] = aa;
      B[r] = bb;
      sa += aa;
      sb += bb;
    }
  }
  if (lane == 0) {
    red[0][warp] = sa;
    red[1][warp] = sb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < 8; ++w) {
      ta += red[0][w];
      tb += red[1][w];
    }
    partial[2 * blockIdx.x] = ta;
    partial[2 * blockIdx.x + 1] = tb;
  }
}

// e_j and the per-column/per-row constants of the filter. Slack factors: the f32 sums of n, A, B
// are inflated by 2^-16 relative; gamma covers the reference's own f32 distance sum, every f32
// rounding of the epilogue and of these constants.
//
// The filter's accumulator starts at -g_j / 2 (a rank-1 MMA: ones x the column term gq) and adds
// h_i . h_j on top, so its rounding also sees the column term: every one of the S = KP/16 + 1 MMA steps
// may lose 17 * 2^-21 of the largest magnitude in the sum, |g_j|/2 + sum_k |h_ik h_jk|; the column
// part goes to e_j, the product part is split by AM-GM like eta. gq[j] stores -g_j / 4 as three bf16
// parts with an exact sum, twice (elements 0..2 and 8..10, zero elsewhere), so that the all-ones row
// operand sums them to -g_j / 2 whatever the swizzle order of the two 16-byte halves.
__global__ void bound_kernel(uint64_t n, uint64_t n_pad, int d, int KP, float rho, const float* __restrict__ nrm,
                             const float* __restrict__ A, const float* __restrict__ B, float2* __restrict__ ge,
                             uint16_t* __restrict__ gq, uint32_t* __restrict__ e4max_bits) {
  const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= n_pad) return;
  uint16_t parts[3] = {0, 0, 0};
  if (j >= n) {
    ge[j] = make_float2(__int_as_float(0x7f800000), 0.0f);  // +inf: padding columns never pass
    parts[0] = 0xFF80u;                                       // bf16 -inf: D = -inf, v = +inf
  } else {
    const float infl = 1.0f + 1.52587890625e-05f;  // 1 + 2^-16
    const float a = A[j] * infl, b = B[j] * infl, nn = nrm[j] * infl;
    const float eta = static_cast<float>(KP) * 4.76837158203125e-07f;                  // K * 2^-21
    const float eta_s = static_cast<float>(KP / 16 + 1) * 17.0f * 4.76837158203125e-07f;  // S * 17 * 2^-21
    // f32 sums of n (d terms), the reference's own distance sum (d/8 + 8 terms, on D <= 2(n_i + n_j)),
    // and the epilogue's roundings: (2d + 64) 2^-24 + 2^-19.
    const float gamma = static_cast<float>(2 * d + 64) * 5.9604644775390625e-08f + 1.9073486328125e-06f;
    const float e0 = 0.5f * (rho * a + b / rho) + 0.5f * b + 0.5f * eta * a + gamma * nn;
    const float e = e0 + 0.5f * eta_s * a + 0.5f * eta_s * (nn + 4.0f * e0) + 1e-30f;
    const float e_safe = e * (1.0f + 9.765625e-04f);  // 2^-10 relative margin on the bound itself
    const float g = nrm[j] - 2.0f * e_safe;
    ge[j] = make_float2(g, 4.0f * e_safe);
    atomicMax(e4max_bits, __float_as_uint(4.0f * e_safe));  // non-negative floats order as their bits
    const float q = -0.25f * g;
    const __nv_bfloat16 p0 = __float2bfloat16_rn(q);
    const float r1 = q - __bfloat162float(p0);
    const __nv_bfloat16 p1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 p2 = __float2bfloat16_rn(r1 - __bfloat162float(p1));
    parts[0] = __bfloat16_as_ushort(p0);
    parts[1] = __bfloat16_as_ushort(p1);
    parts[2] = __bfloat16_as_ushort(p2);
  }
  uint4 w[2];
  w[0] = make_uint4(parts[0] | (static_cast<uint32_t>(parts[1]) << 16), parts[2], 0u, 0u);
  w[1] = w[0];
  reinterpret_cast<uint4*>(gq + j * 16)[0] = w[0];
  reinterpret_cast<uint4*>(gq + j * 16)[1] = w[1];
}

// ---------------------------------------------------------------------------------------------
// 2. the tcgen05 filter
// ---------------------------------------------------------------------------------------------
// Failure-detection test hook (pacmap_debug_stall_knn_loads): when non-zero, the filter's TMA producer
// issues no load and raises nothing itself, so the MMA warp's bounded wait on the operands runs out
// (2 s), raises DEV_ERR_TIMEOUT and aborts the block -- the path a lost copy would take. Zero otherwise.
__device__ int g_debug_stall_loads = 0;

// K blocks of 64 elements: KP = 64 * KB (KB = 0: run-time kb_rt, MODE_STREAM only); candidate buffer
// C = 32 * PER per row.
template <int KB, int PER, int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1) knn_filter_kernel(
    const __grid_constant__ CUtensorMap hmap, const __grid_constant__ CUtensorMap gmap, uint64_t n, uint64_t n_pad,
    int kb_rt, uint32_t idesc, const float2* __restrict__ ge, const float* __restrict__ nrm,
    const uint32_t* __restrict__ perm, int rank, uint2* __restrict__ cand, int* __restrict__ cand_cnt,
    uint32_t* __restrict__ overflow_rows, uint32_t* __restrict__ n_overflow, uint32_t* __restrict__ err,
    int block_offset, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_list,
    const float* __restrict__ resume_theta, const uint32_t* __restrict__ e4max_bits,
    unsigned long long* __restrict__ counters) {
  using L = FilterLayout<KB, MODE>;
  constexpr int NST = L::NST;
  constexpr int C = 32 * PER;
  const int nkb = KB > 0 ? KB : kb_rt;
  const int nch = MODE == MODE_TILE ? 1 : nkb;  // stages per column tile
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  // 1024-byte aligned operand region: resident A [2 halves][KB][16 KB] (not in MODE_STREAM), the
  // all-ones tile [4 KB], the column-term tiles [NST][4 KB], the stages [NST][L::STAGE], then TcShared.
  // Inside a stage: the column tile's K block(s) first, then (MODE_STREAM) the two A halves' K block.
  // aligned by offsetting the shared array itself, so every access keeps the shared address space
  unsigned char* base = tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u);
  unsigned char* a_smem = base;
  unsigned char* one_smem = base + L::A_RES;
  unsigned char* g_smem = one_smem + G_BYTES;
  unsigned char* st_smem = g_smem + NST * G_BYTES;
  TcShared* sh = reinterpret_cast<TcShared*>(st_smem + NST * L::STAGE);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = static_cast<int>(blockIdx.x) + block_offset;  // row block (a shard runs a range of them)
  const uint64_t row0 = static_cast<uint64_t>(blk) * TC_BM;
  const int ntiles = static_cast<int>(n_pad / TC_BN);
  // the column tiles this block visits: all of them in the sweep order, or (approximate kNN) its list
  const uint32_t lbase = tile_ptr ? tile_ptr[blk] : 0u;
  const int nt = tile_ptr ? static_cast<int>(tile_ptr[blk + 1] - lbase) : ntiles;
  auto tile_at = [&](int t) -> int {
    return tile_ptr ? static_cast<int>(tile_list[lbase + t]) : sweep_tile(t, blk, ntiles);
  };

  // A operand of the column-term MMA: bf16 1.0 in every element (every swizzle reads the same tile).
  for (int e = threadIdx.x; e < G_BYTES / 4; e += TC_THREADS) reinterpret_cast<uint32_t*>(one_smem)[e] = 0x3F803F80u;
  fence_proxy_async_smem();
  if (threadIdx.x == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(&sh->full[q], 1);
      mbar_init(&sh->empty[q], 1);
    }
    mbar_init(&sh->a_full, 1);
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sh->tmem_full[a], 1);
      mbar_init(&sh->tmem_empty[a], TC_EPI_WARPS);
    }
    mbar_init(&sh->mma_done, 1);
    sh->abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;
  volatile int* abort_flag = &sh->abort_flag;

  if (warp == 0) {
    // ------------------------------- TMA producer -------------------------------
    if (lane == 0) {
      const bool stall = *reinterpret_cast<volatile int*>(&g_debug_stall_loads) != 0;
      const bool a_issued = MODE != MODE_STREAM && !stall;
      if (a_issued) {
        mbar_expect_tx(&sh->a_full, L::A_RES);
        for (int h = 0; h < 2; ++h)
          for (int kb = 0; kb < KB; ++kb)
            tma_load_2d(a_smem + (h * KB + kb) * KB_BYTES, &hmap, &sh->a_full, kb * 64, static_cast<int>(row0 + h * 128));
      }
      const int total = nt * nch;
      int issued = 0, s = 0, ph = 0;
      bool stop = false;
      for (int t = 0; t < nt && !stop && !stall; ++t) {
        const int tile = tile_at(t);
        for (int ch = 0; ch < nch; ++ch) {
          if (issued >= NST && !mbar_wait(&sh->empty[s], ph ^ 1, abort_flag)) {
            stop = true;
            break;
          }
          unsigned char* st = st_smem + s * L::STAGE;
          const uint32_t bytes = (MODE == MODE_TILE ? KB * KB_BYTES : KB_BYTES) +
                                 (MODE == MODE_STREAM ? 2 * KB_BYTES : 0) + (ch == 0 ? G_BYTES : 0);
          mbar_expect_tx(&sh->full[s], bytes);
          if (MODE == MODE_TILE) {
            for (int kb = 0; kb < KB; ++kb) tma_load_2d(st + kb * KB_BYTES, &hmap, &sh->full[s], kb * 64, tile * TC_BN);
          } else {
            tma_load_2d(st, &hmap, &sh->full[s], ch * 64, tile * TC_BN);
            if (MODE == MODE_STREAM)
              for (int h = 0; h < 2; ++h)
                tma_load_2d(st + (1 + h) * KB_BYTES, &hmap, &sh->full[s], ch * 64, static_cast<int>(row0 + h * 128));
          }
          if (ch == 0) tma_load_2d(g_smem + s * G_BYTES, &gmap, &sh->full[s], 0, tile * TC_BN);
          ++issued;
          if (++s == NST) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if (issued < total && !stall) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      // Drain: every issued load has landed before the block may exit (bounded, whatever the abort flag).
      if (a_issued) {
        const uint64_t t0 = globaltimer();
        while (!mbar_try_wait(&sh->a_full, 0) && globaltimer() - t0 < WAIT_LIMIT_NS) {
        }
      }
      for (int q = (issued > NST ? issued - NST : 0); q < issued; ++q) {
        const uint64_t t0 = globaltimer();
        while (!mbar_try_wait(&sh->full[q % NST], (q / NST) & 1) && globaltimer() - t0 < WAIT_LIMIT_NS) {
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------- MMA issuer -------------------------------
    if (lane == 0) {
      bool ok = MODE == MODE_STREAM ? true : mbar_wait(&sh->a_full, 0, abort_flag);
      const uint32_t a_addr = smem_u32(a_smem), st_addr = smem_u32(st_smem), g_addr = smem_u32(g_smem);
      const uint64_t ones = sdesc_sw32(smem_u32(one_smem));
      const uint32_t idesc_col = idesc_f16(true);  // the column term is bf16 x bf16
      int s = 0, ph = 0;
      for (int t = 0; ok && t < nt; ++t) {
        const int acc = t & 1;
        for (int ch = 0; ch < nch; ++ch) {
          if (!mbar_wait(&sh->full[s], ph, abort_flag)) {
            ok = false;
            break;
          }
          if (ch == 0 && t >= 2 && !mbar_wait(&sh->tmem_empty[acc], ((t >> 1) + 1) & 1, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = st_addr + s * L::STAGE;
          const uint64_t gd = sdesc_sw32(g_addr + s * G_BYTES);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t d_tmem = tmem + acc * 256 + h * 128;
            // D = -g_j / 2 (rank-1: ones x the column term), then D += h_i . h_j over the K blocks in order
            if (ch == 0) umma_f16(d_tmem, ones, gd, idesc_col, 0u);
            if (MODE == MODE_TILE) {
#pragma unroll
              for (int kb = 0; kb < KB; ++kb) {
                const uint64_t ad = sdesc_sw128(a_addr + (h * KB + kb) * KB_BYTES);
                const uint64_t bd = sdesc_sw128(st + kb * KB_BYTES);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) umma_f16(d_tmem, ad + 2 * kk, bd + 2 * kk, idesc, 1u);
              }
            } else {
              const uint64_t ad = sdesc_sw128(MODE == MODE_STREAM ? st + (1 + h) * KB_BYTES
                                                                  : a_addr + (h * KB + ch) * KB_BYTES);
              const uint64_t bd = sdesc_sw128(st);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) umma_f16(d_tmem, ad + 2 * kk, bd + 2 * kk, idesc, 1u);
            }
          }
          umma_commit(&sh->empty[s]);
          if (++s == NST) {
            s = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        umma_commit(&sh->tmem_full[acc]);
      }
      if (!ok) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      // Every issued MMA has completed before the tensor memory is released.
      umma_commit(&sh->mma_done);
      const uint64_t t0 = globaltimer();
      while (!mbar_try_wait(&sh->mma_done, 0) && globaltimer() - t0 < WAIT_LIMIT_NS) {
      }
    }
  } else {
    // ------------------------------- epilogue (8 warps) -------------------------------
    // The accumulator holds D = h_i . h_j - g_j / 2, so v_ij = g_j - 2 G_ij = -2 D exactly; a
    // column passes when v <= theta. Each 32-column group is screened by its maximum D first.
    const int ew = warp - 2;
    const int half = ew >> 2;
    const int quad = warp & 3;  // TMEM lane quadrant this warp may access
    const uint64_t row = row0 + half * 128 + quad * 32 + lane;
    const bool valid = row < n;
    float theta = valid ? 3.402823466e+38f : -__int_as_float(0x7f800000);
    int cnt = 0;
    if (resume_theta && valid) {
      // continue from an earlier pass over other tiles: its compacted buffer and threshold (an overflowed
      // row stays overflowed; it is already listed for the exact fallback)
      const int c0 = cand_cnt[row];
      if (c0 < 0) {
        theta = -__int_as_float(0x7f800000);
      } else {
        cnt = c0;
        theta = resume_theta[row];
      }
    }
    const float n_i = valid ? nrm[row] : 0.0f;
    const float e4_i = valid ? ge[row].y : 0.0f;
    const uint64_t cbase = row * static_cast<uint64_t>(C);
    const float e4max = __uint_as_float(*e4max_bits);
    bool ok = true;
    uint32_t n_ins = 0, n_comp = 0;  // this row's insertions and compactions (statistics)
    const int cnt0 = cnt;            // entries carried over from an earlier pass
    auto screen = [&](const uint32_t (&r)[32], int colb) {
      const float* Dv = reinterpret_cast<const float*>(r);
      float m8[4];
#pragma unroll
      for (int g = 0; g < 4; ++g)
        m8[g] = fmax3(fmax3(Dv[8 * g], Dv[8 * g + 1], Dv[8 * g + 2]), fmax3(Dv[8 * g + 3], Dv[8 * g + 4], Dv[8 * g + 5]),
                      fmaxf(Dv[8 * g + 6], Dv[8 * g + 7]));
      const float m = fmaxf(fmax3(m8[0], m8[1], m8[2]), m8[3]);
      // v = -2 D <= theta exactly when D >= -theta / 2 (both scalings by 2 are exact)
      const float hth = -0.5f * theta;
      if (__any_sync(0xFFFFFFFFu, m >= hth)) {
        // every column of the 32 without a branch: a predicated store of (j, v = -2 D) that also returns the
        // count (a divergent branch per column, or a vote per 8 columns, cost more than the column's work)
#pragma unroll
        for (int c = 0; c < 32; ++c)
          cnt += st_global_v2_if_ge(cand + cbase + cnt, static_cast<uint32_t>(colb + c), __float_as_uint(-2.0f * Dv[c]),
                                    Dv[c], hth);
      }
    };
    for (int t = 0; t < nt; ++t) {
      const int acc = t & 1;
      if (!mbar_wait(&sh->tmem_full[acc], (t >> 1) & 1, abort_flag)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int col0 = tile_at(t) * TC_BN;
      const uint32_t taddr = tmem + (static_cast<uint32_t>(quad * 32) << 16) + acc * 256 + half * 128;
#pragma unroll
      for (int cp = 0; cp < 2; ++cp) {  // 64 columns per pass, two TMEM loads in flight
        uint32_t r0[32], r1[32];
        tmem_ld32_issue(taddr + cp * 64, r0);
        tmem_ld32_issue(taddr + cp * 64 + 32, r1);
        tmem_wait_ld_tied(r0);
        tie_regs(r1);
        screen(r0, col0 + cp * 64);
        screen(r1, col0 + cp * 64 + 32);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh->tmem_empty[acc]);
      // Compact full buffers so that the next tile (<= 128 insertions) always fits.
      // The next row's entries are loaded before the current row is compacted (their latency overlaps).
      unsigned need = __ballot_sync(0xFFFFFFFFu, cnt > C - TC_BN);
      if (need) {
        int L = __ffs(need) - 1;
        need &= need - 1;
        RowRegs<PER> cur;
        load_row<PER>(cand + __shfl_sync(0xFFFFFFFFu, cbase, L), __shfl_sync(0xFFFFFFFFu, cnt, L), cur);
        while (true) {
          // PER > 16 keeps one row in registers at a time (two would spill)
          const int L2 = need ? __ffs(need) - 1 : -1;
          RowRegs<PER> nxt;
          if (PER <= 16 && L2 >= 0)
            load_row<PER>(cand + __shfl_sync(0xFFFFFFFFu, cbase, L2), __shfl_sync(0xFFFFFFFFu, cnt, L2), nxt);
          const uint64_t rb = __shfl_sync(0xFFFFFFFFu, cbase, L);
          const int m = __shfl_sync(0xFFFFFFFFu, cnt, L);
          const float nL = __shfl_sync(0xFFFFFFFFu, n_i, L);
          const float eL = __shfl_sync(0xFFFFFFFFu, e4_i, L);
          float th;
          // gather-free first (theta from the largest e); only when its band would not fit, again with every
          // entry's own e_j (the band holds the rank entries of smallest u, so the tighter theta is the
          // whole buffer's)
          const float thL = __shfl_sync(0xFFFFFFFFu, theta, L);
          int kept = compact_row<PER>(cand + rb, m, min(rank, m), nL, eL, cur, e4max, nullptr, thL, th, nullptr,
                                      FILTER_SLACK);
          if (kept > C - TC_BN) kept = recompact_exact<PER>(cand + rb, kept, rank, nL, eL, ge, th, th);
          if (lane == L) {
            theta = th;
            cnt = kept;
            ++n_comp;
            if (cnt > C - TC_BN) {  // the band does not fit: exact recomputation later
              theta = -__int_as_float(0x7f800000);
              cnt = 0;
              overflow_rows[atomicAdd(n_overflow, 1u)] = perm[row];
            }
            n_ins += static_cast<uint32_t>(m - cnt);  // the entries this compaction dropped
          }
          __syncwarp();
          if (L2 < 0) break;
          need &= need - 1;
          L = L2;
          if (PER <= 16) cur = nxt;
          else load_row<PER>(cand + __shfl_sync(0xFFFFFFFFu, cbase, L), __shfl_sync(0xFFFFFFFFu, cnt, L), cur);
        }
      }
    }
    if (!ok) {
      atomicOr(err, DEV_ERR_TIMEOUT);
      sh->abort_flag = 1;
    }
    if (valid) cand_cnt[row] = (theta == -__int_as_float(0x7f800000)) ? -1 : cnt;
    n_ins += static_cast<uint32_t>(cnt - cnt0);  // dropped + left = inserted + present at the start
    if (counters) {
      const uint32_t wi = __reduce_add_sync(0xFFFFFFFFu, n_ins), wc = __reduce_add_sync(0xFFFFFFFFu, n_comp);
      if (lane == 0) {
        atomicAdd(&counters[0], static_cast<unsigned long long>(wi));
        atomicAdd(&counters[1], static_cast<unsigned long long>(wc));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------------------------
// 3. exact re-rank: one warp per (permuted) row; output at the original row, original indices.
// ---------------------------------------------------------------------------------------------
// 3a. final compaction: the row's certified band (v <= theta of its rank-th upper bound), one warp
//     per row; the count is written back (rows that overflowed in the filter keep -1).
//     With ub (the tile pruning's first pass): ub[r] = an upper bound at or above the rank-th smallest upper
//     bound of the reference's squared distance (scaled by s^2) over the columns the row met, u + n_i + 2 e_i
//     rounded up -- an upper bound of its k'-th neighbour distance, since k' of those rank columns are
//     other points;
//     +inf when the row met fewer than rank columns or overflowed.
constexpr int RC_WARPS = 4;

template <int PER>
__global__ void __launch_bounds__(RC_WARPS * 32) knn_compact_kernel(
    uint64_t n, int rank, const float* __restrict__ nrm, const float2* __restrict__ ge, uint2* __restrict__ cand,
    int* __restrict__ cand_cnt, float* __restrict__ ub, float* __restrict__ theta_out,
    unsigned long long* __restrict__ band_total) {
  constexpr int C = 32 * PER;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned long long band = 0;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * RC_WARPS + warp; r < n;
       r += static_cast<uint64_t>(gridDim.x) * RC_WARPS) {
    const int m0 = min(cand_cnt[r], C);
    if (m0 <= 0 || (ub && m0 < rank)) {
      if (ub && lane == 0) ub[r] = __int_as_float(0x7f800000);
      if (theta_out && lane == 0) theta_out[r] = 3.402823466e+38f;  // every column met is still kept
      continue;
    }
    const uint64_t rb = r * static_cast<uint64_t>(C);
    float th;
    uint32_t ukey = 0;
    const float n_i = nrm[r], e4_i = ge[r].y;
    RowRegs<PER> regs;
    load_row<PER>(cand + rb, m0, regs);
    // the early exit leaves ukey at or above the rank-th smallest upper bound: ub and theta stay valid
    // bounds and the band a superset of the exact one (the re-rank's result is the same)
    const int m = compact_row<PER>(cand + rb, m0, min(rank, m0), n_i, e4_i, regs, 0.0f, ge, 3.402823466e+38f, th,
                                   &ukey, FILTER_SLACK);
    band += static_cast<unsigned long long>(m);
    if (lane == 0) {
      cand_cnt[r] = m;
      if (theta_out) theta_out[r] = th;
      if (ub) {
        // two f32 additions: within 2^-23 of the magnitudes summed (rounded up by 2^-22 of them)
        const float uk = key_to_float(ukey);
        const float u = (uk + n_i + 0.5f * e4_i) + 2.384185791015625e-07f * (fabsf(uk) + n_i + e4_i);
        ub[r] = (u >= 0.0f && u <= 3.4e38f) ? u : __int_as_float(0x7f800000);
      }
    }
  }
  if (band_total && lane == 0 && band) atomicAdd(band_total, band);
}

// 3b. exact re-rank of the compacted band: the reference's f32 distance of every survivor (8-lane
//     groups in distance.rs:50-75's lane order, each lane reading its terms four at a time from the
//     lane-grouped rows, 4 survivors per warp pass, row i of x in registers when it has at most 4 NQ
//     chunks of 8, else read from L1 each pass with NQ = 0), sorted by (distance, index); output at the
//     original row, original indices.
// x: the rows in the locality order (row r is point perm[r]) in RerankLayout; candidates of nearby rows
// sit nearby.
__device__ __forceinline__ float add_sq4(float acc, const float4 a, const float4 b) {
  const float d0 = __fsub_rn(a.x, b.x), d1 = __fsub_rn(a.y, b.y), d2 = __fsub_rn(a.z, b.z), d3 = __fsub_rn(a.w, b.w);
  acc = __fadd_rn(acc, __fmul_rn(d0, d0));
  acc = __fadd_rn(acc, __fmul_rn(d1, d1));
  acc = __fadd_rn(acc, __fmul_rn(d2, d2));
  return __fadd_rn(acc, __fmul_rn(d3, d3));
}
__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

template <int PER, int WARPS, int NQ>
__global__ void __launch_bounds__(WARPS * 32) knn_rerank_kernel(
    const float* __restrict__ x, uint64_t n, int d, int K, const uint32_t* __restrict__ perm,
    const uint2* __restrict__ cand, const int* __restrict__ cand_cnt, uint32_t* __restrict__ out_idx,
    float* __restrict__ out_dist, uint32_t* __restrict__ fallback_rows, uint32_t* __restrict__ n_fallback) {
  constexpr int C = 32 * PER;
  __shared__ uint64_t keys_all[WARPS][C];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* keys = keys_all[warp];
  const int l8 = lane & 7, grp = lane >> 3;
  const RerankLayout lay = rerank_layout(d);
  const int nq = lay.nq, tail0 = 32 * lay.nq;
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * WARPS + warp; r < n;
       r += static_cast<uint64_t>(gridDim.x) * WARPS) {
    const int m = min(cand_cnt[r], C);
    if (m < 0) continue;  // overflowed in the filter: handled by the exact fallback
    const uint64_t rb = r * static_cast<uint64_t>(C);
    const uint64_t orow = perm[r];
    const float* a = x + r * lay.ds;
    float4 ra[NQ > 0 ? NQ : 1];
#pragma unroll
    for (int k = 0; k < NQ; ++k) ra[k] = k < nq ? ld4(a + 32 * k + 4 * l8) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int nk = 0;
    // 32 candidates per chunk: their indices and original ids by one coalesced and one parallel load, then
    // two candidates per 8-lane group and pass, both rows' loads issued before either sum
    for (int c0 = 0; c0 < m; c0 += 32) {
      const bool mine = c0 + lane < m;
      const uint32_t my_jp = mine ? cand[rb + c0 + lane].x : static_cast<uint32_t>(r);
      const uint32_t my_j = perm[my_jp];
      const int span = min(32, m - c0);
      for (int q0 = 0; q0 < span; q0 += 8) {
        float t2[2];
        uint32_t jp2[2], j2[2];
        bool real2[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = q0 + 4 * h + grp;  // 0..31 within the chunk
          jp2[h] = __shfl_sync(0xFFFFFFFFu, my_jp, q & 31);
          j2[h] = __shfl_sync(0xFFFFFFFFu, my_j, q & 31);
          real2[h] = (q < span) && (jp2[h] != r);
        }
        const float* b0 = x + static_cast<uint64_t>(jp2[0]) * lay.ds;
        const float* b1 = x + static_cast<uint64_t>(jp2[1]) * lay.ds;
        float acc0 = 0.0f, acc1 = 0.0f;
        if (NQ > 0) {
          float4 v0[NQ > 0 ? NQ : 1], v1[NQ > 0 ? NQ : 1];
#pragma unroll
          for (int k = 0; k < NQ; ++k) {
            if (k < nq) {
              v0[k] = ld4(b0 + 32 * k + 4 * l8);
              v1[k] = ld4(b1 + 32 * k + 4 * l8);
            }
          }
#pragma unroll
          for (int k = 0; k < NQ; ++k) {
            if (k < nq) {
              acc0 = add_sq4(acc0, ra[k], v0[k]);
              acc1 = add_sq4(acc1, ra[k], v1[k]);
            }
          }
        } else {
          for (int k = 0; k < nq; ++k) {
            const float4 av = ld4(a + 32 * k + 4 * l8);
            acc0 = add_sq4(acc0, av, ld4(b0 + 32 * k + 4 * l8));
            acc1 = add_sq4(acc1, av, ld4(b1 + 32 * k + 4 * l8));
          }
        }
        t2[0] = 0.0f;
        t2[1] = 0.0f;
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          t2[0] = __fadd_rn(t2[0], __shfl_sync(0xFFFFFFFFu, acc0, (lane & ~7) + l));
          t2[1] = __fadd_rn(t2[1], __shfl_sync(0xFFFFFFFFu, acc1, (lane & ~7) + l));
        }
        for (int q = 0; q < lay.tail; ++q) {
          const float av = a[tail0 + q];
          const float d0 = __fsub_rn(av, b0[tail0 + q]), d1 = __fsub_rn(av, b1[tail0 + q]);
          t2[0] = __fadd_rn(t2[0], __fmul_rn(d0, d0));
          t2[1] = __fadd_rn(t2[1], __fmul_rn(d1, d1));
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float dist = __fsqrt_rn(t2[h]);
          const unsigned bal = __ballot_sync(0xFFFFFFFFu, real2[h] && l8 == 0);
          if (real2[h] && l8 == 0) {
            const int pos = nk + __popc(bal & ((1u << lane) - 1u));
            keys[pos] = (static_cast<uint64_t>(total_key(dist)) << 32) | j2[h];
          }
          nk += __popc(bal);
        }
      }
    }
    __syncwarp();
    if (nk < K) {  // fewer certified candidates than neighbours (non-finite data): exact fallback
      if (lane == 0) fallback_rows[atomicAdd(n_fallback, 1u)] = static_cast<uint32_t>(orow);
      __syncwarp();
      continue;
    }
    if (nk <= 128) {  // sorted in registers: up to 4 keys per lane
      auto sort_regs = [&](auto tag) {
        constexpr int R = decltype(tag)::value;
        uint64_t v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int e = r * 32 + lane;
          v[r] = e < nk ? keys[e] : ~0ull;
        }
        warp_sort_regs_u64<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int c = r * 32 + lane;
          if (c < K) {
            out_idx[orow * K + c] = static_cast<uint32_t>(v[r] & 0xFFFFFFFFu);
            out_dist[orow * K + c] = key_to_float(static_cast<uint32_t>(v[r] >> 32));
          }
        }
      };
      if (nk <= 32) sort_regs(std::integral_constant<int, 1>());
      else if (nk <= 64) sort_regs(std::integral_constant<int, 2>());
      else sort_regs(std::integral_constant<int, 4>());
      __syncwarp();
      continue;
    }
    const int Pr = next_pow2(nk);
    for (int e = nk + lane; e < Pr; e += 32) keys[e] = ~0ull;
    warp_bitonic_sort_u64(keys, Pr);
    for (int c = lane; c < K; c += 32) {
      const uint64_t kv = keys[c];
      out_idx[orow * K + c] = static_cast<uint32_t>(kv & 0xFFFFFFFFu);
      out_dist[orow * K + c] = key_to_float(static_cast<uint32_t>(kv >> 32));
    }
    __syncwarp();
  }
}

}  // namespace

bool knn_tc_supported(uint64_t n, uint64_t d, uint64_t kp) {
  return d >= 1 && d <= 1024 && kp >= 1 && kp + 1 <= 448 && n >= 2 && n < (1ull << 31);
}

// The pivots' rows into a PIV x d array.
__global__ void gather_pivots_kernel(const float* __restrict__ x, const uint32_t* __restrict__ piv_rows, int d,
                                     float* __restrict__ out) {
  const int p = blockIdx.x;
  const uint64_t row = piv_rows[p];
  for (int c = threadIdx.x; c < d; c += blockDim.x) out[static_cast<uint64_t>(p) * d + c] = x[row * d + c];
}

__global__ void mark_owned_kernel(const uint32_t* __restrict__ perm, uint64_t r0, uint64_t r1,
                                  uint8_t* __restrict__ owned) {
  const uint64_t r = r0 + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r < r1) owned[perm[r]] = 1;
}

bool knn_tc_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, bool bf16, uint32_t* d_idx,
                   float* d_dist, const KnnShard& shard, int nprobe, bool prune) {
  if (!knn_tc_supported(n, d, kp)) return false;
  KnnTcStats& st = last_tc_stats();
  st = KnnTcStats();
  const int KB = static_cast<int>((d + 63) / 64);
  const int KP = 64 * KB;
  const int mode = KB <= 2 ? MODE_TILE : (KB <= 4 ? MODE_KBLOCK : MODE_STREAM);
  const uint64_t n_pad = (n + TC_BM - 1) / TC_BM * TC_BM;
  const uint64_t nblocks = n_pad / TC_BM, ntl = n_pad / TC_BN;
  const int PER = (kp + 1 <= 192) ? 16 : 32;  // buffer C = 512 or 1024 candidates per row
  const int C = 32 * PER;
  const int rank = static_cast<int>(kp) + 1;
  // Tile pruning pays once the tiles are many; its lists are indexed with 32 bits.
  prune = prune && nprobe == 0 && n >= PRUNE_MIN_ROWS && nblocks * ntl < (1ull << 32);

  // scale: an exact power of two with max |x s| < 2^13
  DevBuf<uint32_t> amax(c, 1);
  PM_CUDA(cudaMemsetAsync(amax.get(), 0, sizeof(uint32_t), c.stream));
  absmax_kernel<<<std::min<unsigned>(ceil_div(n * d, 256), c.sm_count * 8), 256, 0, c.stream>>>(d_x, n * d, amax.get());
  PM_LAUNCHED();
  uint32_t hbits = 0;
  PM_CUDA(cudaMemcpyAsync(&hbits, amax.get(), 4, cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  float amx;
  std::memcpy(&amx, &hbits, 4);
  if (!(amx > 0.0f) || !std::isfinite(amx)) return false;  // all-zero or non-finite data: SIMT path
  int ex = 0;
  std::frexp(amx, &ex);  // amx in [2^(ex-1), 2^ex)
  const float s = std::ldexp(1.0f, 13 - ex);

  // locality order: pivots by k-means++ seeding, every point to its nearest pivot, a stable sort by cell
  const uint32_t chunks = ceil_div(n, PL_CHUNK);
  DevBuf<uint32_t> piv_rows(c, PIV), cell(c, n), cell_counts(c, static_cast<uint64_t>(chunks) * PIV), perm(c, n);
  select_pivots(c, d_x, n, d, piv_rows.get());
  DevBuf<float> score, pnorm;
  if (prune) {
    score.alloc(c, n * PIV);
    pnorm.alloc(c, PIV);
  }
  const int dpad = static_cast<int>((d + PA_D - 1) / PA_D * PA_D);
  DevBuf<float> pT(c, static_cast<uint64_t>(dpad) * PIV);
  pivots_t_kernel<<<ceil_div(static_cast<uint64_t>(dpad) * PIV, 256), 256, 0, c.stream>>>(d_x, piv_rows.get(),
                                                                                          static_cast<int>(d), dpad,
                                                                                          pT.get());
  PM_LAUNCHED();
  pivot_assign_kernel<<<ceil_div(n, PA_PTS), 256, 0, c.stream>>>(d_x, n, static_cast<int>(d), pT.get(), cell.get(),
                                                                 score.get(), pnorm.get());
  PM_LAUNCHED();
  cell_chunk_count_kernel<<<chunks, 256, 0, c.stream>>>(cell.get(), n, cell_counts.get());
  PM_LAUNCHED();
  cell_chunk_offsets_kernel<<<1, PIV, 0, c.stream>>>(cell_counts.get(), chunks);
  PM_LAUNCHED();
  cell_place_kernel<<<chunks, 32, 0, c.stream>>>(cell.get(), n, cell_counts.get(), perm.get());
  PM_LAUNCHED();

  // Tile lists over the cells nearest each row block: every row block visits only the column tiles of
  // the `probe` pivot cells whose pivots are nearest its own cells' (own cells first). The cells are
  // contiguous ranges of the locality order: cell p starts at the first chunk's offset for p.
  const uint64_t blocks_all = nblocks;
  const uint64_t sblk0 = blocks_all * shard.index / shard.count, sblk1 = blocks_all * (shard.index + 1) / shard.count;
  auto probe_lists = [&](int probe, uint32_t min_cell, DevBuf<uint32_t>& tile_ptr,
                         DevBuf<uint32_t>& tile_list) -> uint64_t {
    if (ntl <= 131072)  // on the device: the cell starts are the first chunk's offsets
      return build_probe_tile_lists(c, d_x, d, piv_rows.get(), cell_counts.get(), n, n_pad, probe, min_cell, sblk0,
                                    sblk1, tile_ptr, tile_list);
    std::vector<uint32_t> cstart(PIV + 1);
    DevBuf<float> piv(c, static_cast<uint64_t>(PIV) * d);
    gather_pivots_kernel<<<PIV, 128, 0, c.stream>>>(d_x, piv_rows.get(), static_cast<int>(d), piv.get());
    PM_LAUNCHED();
    std::vector<float> hp(static_cast<size_t>(PIV) * d);
    PM_CUDA(cudaMemcpyAsync(cstart.data(), cell_counts.get(), PIV * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(hp.data(), piv.get(), hp.size() * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    cstart[PIV] = static_cast<uint32_t>(n);
    // nearest pivots of each pivot (itself first), by f64 squared distance, ties to the lower index
    std::vector<std::vector<int>> near(PIV);
    std::vector<std::pair<double, int>> dd(PIV);
    for (int p = 0; p < PIV; ++p) {
      for (int q = 0; q < PIV; ++q) {
        double acc = 0.0;
        for (uint64_t k = 0; k < d; ++k) {
          const double df = static_cast<double>(hp[p * d + k]) - hp[q * d + k];
          acc += df * df;
        }
        dd[q] = {q == p ? -1.0 : acc, q};
      }
      std::partial_sort(dd.begin(), dd.begin() + probe, dd.end());
      for (int r = 0; r < probe; ++r) near[p].push_back(dd[r].second);
    }
    std::vector<uint32_t> ptr(nblocks + 1, 0), list;
    std::vector<uint64_t> stamp(ntl, ~0ull);
    list.reserve(nblocks * static_cast<uint64_t>(probe) * 40);
    auto add_cell = [&](int q, uint64_t b) {
      if (cstart[q + 1] <= cstart[q]) return;
      for (uint64_t t = cstart[q] / TC_BN; t <= (cstart[q + 1] - 1) / TC_BN; ++t)
        if (stamp[t] != b) {
          stamp[t] = b;
          list.push_back(static_cast<uint32_t>(t));
        }
    };
    for (uint64_t b = 0; b < nblocks; ++b) {
      const uint64_t r0 = b * TC_BM, r1 = std::min<uint64_t>(r0 + TC_BM, n);
      std::vector<int> own;
      for (int p = 0; p < PIV && r0 < r1; ++p)
        if (cstart[p] < r1 && cstart[p + 1] > r0) own.push_back(p);
      for (int p : own) add_cell(p, b);
      for (int r = 1; r < probe; ++r)
        for (int p : own) add_cell(near[p][r], b);
      ptr[b + 1] = static_cast<uint32_t>(list.size());
    }
    if (list.empty()) list.push_back(0);
    upload(c, tile_ptr, ptr.data(), ptr.size());
    upload(c, tile_list, list.data(), list.size());
    return static_cast<uint64_t>(ptr[sblk1] - ptr[sblk0]);
  };

  DevBuf<uint32_t> tile_ptr, tile_list;
  if (nprobe > 0 && nprobe < PIV) probe_lists(nprobe, 0xFFFFFFFFu, tile_ptr, tile_list);

  DevBuf<uint16_t> H(c, n_pad * KP);
  DevBuf<float> xperm(c, n * static_cast<uint64_t>(rerank_layout(static_cast<int>(d)).ds));
  DevBuf<float> nrm(c, n_pad), A(c, n_pad), B(c, n_pad);
  DevBuf<float2> ge(c, n_pad);
  DevBuf<uint16_t> gq(c, n_pad * 16);
  const unsigned sgrid = std::min<unsigned>(ceil_div(n_pad, 8), c.sm_count * 8);
  DevBuf<double> partial(c, 2 * sgrid);
  if (bf16)
    split_rows_kernel<true><<<sgrid, 256, 0, c.stream>>>(d_x, perm.get(), n, static_cast<int>(d), KP, n_pad, s, H.get(),
                                                       nrm.get(), A.get(), B.get(), partial.get(), xperm.get());
  else
    split_rows_kernel<false><<<sgrid, 256, 0, c.stream>>>(d_x, perm.get(), n, static_cast<int>(d), KP, n_pad, s, H.get(),
                                                        nrm.get(), A.get(), B.get(), partial.get(), xperm.get());
  PM_LAUNCHED();
  std::vector<double> hpart(2 * sgrid);
  PM_CUDA(cudaMemcpyAsync(hpart.data(), partial.get(), hpart.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  double sa = 0.0, sb = 0.0;
  for (unsigned b = 0; b < sgrid; ++b) {
    sa += hpart[2 * b];
    sb += hpart[2 * b + 1];
  }
  const float rho = (sa > 0.0 && sb > 0.0) ? static_cast<float>(std::sqrt(sb / sa)) : 1e-4f;
  DevBuf<uint32_t> e4max(c, 1);
  PM_CUDA(cudaMemsetAsync(e4max.get(), 0, sizeof(uint32_t), c.stream));
  bound_kernel<<<ceil_div(n_pad, 256), 256, 0, c.stream>>>(n, n_pad, static_cast<int>(d), KP, rho, nrm.get(), A.get(),
                                                          B.get(), ge.get(), gq.get(), e4max.get());
  PM_LAUNCHED();

  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(KP), static_cast<cuuint64_t>(n_pad)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(KP) * 2};
  const cuuint32_t box[2] = {64, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult cr = detail::get_encode_fn()(&map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                                      H.get(), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PM_REQUIRE(cr == CUDA_SUCCESS, PACMAP_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(cr));
  // the column term: [n_pad][16] bf16, box 16 x 128, 32-byte swizzle (x is always 0)
  CUtensorMap gmap;
  std::memset(&gmap, 0, sizeof(gmap));
  const cuuint64_t gdims[2] = {16, static_cast<cuuint64_t>(n_pad)};
  const cuuint64_t gstrides[1] = {32};
  const cuuint32_t gbox[2] = {16, 128};
  const CUresult gr = detail::get_encode_fn()(&gmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, gq.get(), gdims, gstrides, gbox,
                                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PM_REQUIRE(gr == CUDA_SUCCESS, PACMAP_ERR_CUDA, "cuTensorMapEncodeTiled (column term) failed: " + std::to_string(gr));

  DevBuf<uint2> cand(c, n_pad * C);
  DevBuf<int> ccnt(c, n_pad);
  // statistics: insertions and compactions of the filter passes, entries of the final bands
  DevBuf<unsigned long long> counters(c, 3);
  PM_CUDA(cudaMemsetAsync(counters.get(), 0, 3 * sizeof(unsigned long long), c.stream));
  DevBuf<uint32_t> ovf(c, n + 1), fbk(c, n + 1);

  const uint32_t idesc = idesc_f16(bf16);
  // this shard's row blocks (in the locality order); the compaction and the re-rank skip the other rows
  const uint64_t blk0 = nblocks * shard.index / shard.count, blk1 = nblocks * (shard.index + 1) / shard.count;
  const unsigned grid = static_cast<unsigned>(blk1 - blk0);
  if (shard.d_owned && blk1 > blk0) {
    const uint64_t r0 = std::min<uint64_t>(blk0 * TC_BM, n), r1 = std::min<uint64_t>(blk1 * TC_BM, n);
    if (r1 > r0) {
      mark_owned_kernel<<<ceil_div(r1 - r0, 256), 256, 0, c.stream>>>(perm.get(), r0, r1, shard.d_owned);
      PM_LAUNCHED();
    }
  }
  // One filter launch over this shard's row blocks: with tile lists (ptr, list) or over every tile.
  auto run_filter = [&](const uint32_t* lptr, const uint32_t* llist, uint32_t* ovf_rows, uint32_t* n_ovf,
                        const float* resume_theta) {
    if (!resume_theta) PM_CUDA(cudaMemsetAsync(ccnt.get(), 0xFF, n_pad * sizeof(int), c.stream));
    auto launch = [&](auto kern, size_t smem) {
      PM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      if (grid == 0) return;
      kern<<<grid, TC_THREADS, smem, c.stream>>>(map, gmap, n, n_pad, KB, idesc, ge.get(), nrm.get(), perm.get(), rank,
                                                 cand.get(), ccnt.get(), ovf_rows, n_ovf, c.d_err,
                                                 static_cast<int>(blk0), lptr, llist, resume_theta, e4max.get(),
                                                 counters.get());
    };
    const bool p16 = PER == 16;
    if (mode == MODE_STREAM) {
      constexpr size_t sm = FilterLayout<0, MODE_STREAM>::SMEM;
      if (p16) launch(knn_filter_kernel<0, 16, MODE_STREAM>, sm);
      else launch(knn_filter_kernel<0, 32, MODE_STREAM>, sm);
    } else if (KB == 1) {
      constexpr size_t sm = FilterLayout<1, MODE_TILE>::SMEM;
      if (p16) launch(knn_filter_kernel<1, 16, MODE_TILE>, sm);
      else launch(knn_filter_kernel<1, 32, MODE_TILE>, sm);
    } else if (KB == 2) {
      constexpr size_t sm = FilterLayout<2, MODE_TILE>::SMEM;
      if (p16) launch(knn_filter_kernel<2, 16, MODE_TILE>, sm);
      else launch(knn_filter_kernel<2, 32, MODE_TILE>, sm);
    } else if (KB == 3) {
      constexpr size_t sm = FilterLayout<3, MODE_KBLOCK>::SMEM;
      if (p16) launch(knn_filter_kernel<3, 16, MODE_KBLOCK>, sm);
      else launch(knn_filter_kernel<3, 32, MODE_KBLOCK>, sm);
    } else {
      constexpr size_t sm = FilterLayout<4, MODE_KBLOCK>::SMEM;
      if (p16) launch(knn_filter_kernel<4, 16, MODE_KBLOCK>, sm);
      else launch(knn_filter_kernel<4, 32, MODE_KBLOCK>, sm);
    }
    PM_LAUNCHED();
  };
  const unsigned cgrid = std::min<unsigned>(ceil_div(n, RC_WARPS), c.sm_count * 16);
  auto compact = [&](float* ub, float* theta_out, unsigned long long* band_total) {
    if (PER == 16)
      knn_compact_kernel<16><<<cgrid, RC_WARPS * 32, 0, c.stream>>>(n, rank, nrm.get(), ge.get(), cand.get(), ccnt.get(),
                                                                    ub, theta_out, band_total);
    else
      knn_compact_kernel<32><<<cgrid, RC_WARPS * 32, 0, c.stream>>>(n, rank, nrm.get(), ge.get(), cand.get(), ccnt.get(),
                                                                    ub, theta_out, band_total);
    PM_LAUNCHED();
  };
  cudaEvent_t ev[3];
  for (auto& e : ev) PM_CUDA(cudaEventCreate(&e));
  PM_CUDA(cudaEventRecord(ev[0], c.stream));
  st.tiles_full = static_cast<uint64_t>(grid) * ntl;
  st.tiles_visited = st.tiles_full;
  PM_CUDA(cudaMemsetAsync(ovf.get() + n, 0, sizeof(uint32_t), c.stream));
  PM_CUDA(cudaMemsetAsync(fbk.get() + n, 0, sizeof(uint32_t), c.stream));
  DevBuf<uint32_t> aptr, alist;
  DevBuf<float> resume;
  if (prune) {
    // First pass: each block over the cells nearest its own gives every row a bound of its k'-th
    // neighbour distance; then the tiles that may hold a neighbour of some row of the block. The second
    // pass continues from the first's compacted buffers and thresholds over the remaining tiles (rows that
    // overflowed in the first pass are already on the exact fallback list).
    // a cell of at least 4 (k'+1) points bounds its rows by itself; smaller cells add their nearest cell
    st.tiles_bound = probe_lists(PRUNE_PROBE, static_cast<uint32_t>(4 * rank), aptr, alist);
    run_filter(aptr.get(), alist.get(), ovf.get(), ovf.get() + n, nullptr);
    c.check_errors("tensor-core kNN bound pass");
    DevBuf<float> ub(c, n_pad);
    resume.alloc(c, n_pad);
    compact(ub.get(), resume.get(), nullptr);
    PruneInputs in;
    in.perm = perm.get();
    in.cell = cell.get();
    in.score = score.get();
    in.pnorm = pnorm.get();
    in.rownorm = nrm.get();
    in.ub = ub.get();
    in.n = n;
    in.n_pad = n_pad;
    in.d = d;
    in.inv_s = 1.0f / s;
    in.blk0 = blk0;
    in.blk1 = blk1;
    in.skip_ptr = aptr.get();
    in.skip_list = alist.get();
    st.tiles_visited = build_pruned_tile_lists(c, in, tile_ptr, tile_list);
  }
  PM_CUDA(cudaEventRecord(ev[1], c.stream));
  run_filter(tile_ptr.get(), tile_list.get(), ovf.get(), ovf.get() + n, prune ? resume.get() : nullptr);
  PM_CUDA(cudaEventRecord(ev[2], c.stream));
  c.check_errors("tensor-core kNN filter");
  float fms = 0.0f, bms = 0.0f;
  PM_CUDA(cudaEventElapsedTime(&bms, ev[0], ev[1]));
  PM_CUDA(cudaEventElapsedTime(&fms, ev[1], ev[2]));
  for (auto& e : ev) cudaEventDestroy(e);
  st.filter_ms = fms;
  st.bound_ms = bms;

  compact(nullptr, nullptr, counters.get() + 2);
  const int di = static_cast<int>(d), ki = static_cast<int>(kp);
  // the re-rank reads xperm with 16-byte loads
  PM_REQUIRE((reinterpret_cast<uintptr_t>(xperm.get()) & 15u) == 0, PACMAP_ERR_CUDA,
             "re-rank copy of x is not 16-byte aligned");
  auto rerank = [&](auto kern, int warps) {
    const unsigned rgrid = std::min<unsigned>(ceil_div(n, warps), c.sm_count * 32);
    kern<<<rgrid, warps * 32, 0, c.stream>>>(xperm.get(), n, di, ki, perm.get(), cand.get(), ccnt.get(), d_idx,
                                             d_dist, fbk.get(), fbk.get() + n);
  };
  // NQ groups of four chunks of 8 in registers: d < 8 * 4 NQ + 8 (the remainder is read separately)
  if (PER == 16) {
    if (d > 256) rerank(knn_rerank_kernel<16, 8, 0>, 8);
    else if (d > 128) rerank(knn_rerank_kernel<16, 8, 8>, 8);
    else if (d > 64) rerank(knn_rerank_kernel<16, 8, 4>, 8);
    else rerank(knn_rerank_kernel<16, 8, 2>, 8);
  } else {
    if (d > 256) rerank(knn_rerank_kernel<32, 4, 0>, 4);
    else if (d > 128) rerank(knn_rerank_kernel<32, 4, 8>, 4);
    else if (d > 64) rerank(knn_rerank_kernel<32, 4, 4>, 4);
    else rerank(knn_rerank_kernel<32, 4, 2>, 4);
  }
  PM_LAUNCHED();

  // Rows the filter could not settle: exact SIMT recomputation, scattered into place.
  uint32_t counts[2] = {0, 0};
  unsigned long long cv[3] = {0, 0, 0};
  PM_CUDA(cudaMemcpyAsync(&counts[0], ovf.get() + n, 4, cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaMemcpyAsync(&counts[1], fbk.get() + n, 4, cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaMemcpyAsync(cv, counters.get(), sizeof(cv), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  st.fallback_rows = counts[0] + counts[1];
  st.insertions = cv[0];
  st.compactions = cv[1];
  st.band_entries = cv[2];
  st.rows = n;
  const uint32_t* lists[2] = {ovf.get(), fbk.get()};
  for (int q = 0; q < 2; ++q) {
    if (!counts[q]) continue;
    knn_rows_simt(c, d_x, n, d, kp, lists[q], counts[q], d_idx, d_dist, /*scatter=*/true);
  }
  return true;
}

KnnTcStats& last_tc_stats() {
  static thread_local KnnTcStats v;
  return v;
}

}  // namespace pacmap

extern "C" pacmap_status pacmap_debug_stall_knn_loads(int32_t device, int32_t on) {
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) {
    cudaGetLastError();
    prev = -1;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    pacmap::set_last_error("no CUDA device is visible");
    return PACMAP_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) {
    pacmap::set_last_error("device ordinal " + std::to_string(device) + " is not available");
    return PACMAP_ERR_INVALID_ARGUMENT;
  }
  const int v = on ? 1 : 0;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pacmap::g_debug_stall_loads, &v, sizeof(int));
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    pacmap::set_last_error(std::string("cudaMemcpyToSymbol: ") + cudaGetErrorString(e));
    return PACMAP_ERR_CUDA;
  }
  pacmap::set_last_error("");
  return PACMAP_OK;
}
