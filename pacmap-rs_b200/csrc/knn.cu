// Exact kNN -- knn::find_k_nearest_neighbors (src/knn.rs:137-194).
//
// The reference forms all n(n-1)/2 upper-triangle f32 distances (knn.rs:149-163), sorts them globally
// (knn.rs:166-167) and fills each row first come, first served (knn.rs:176-191). Row i therefore holds
// its k' = min(k, n-1) smallest distances to j != i in ascending order; ties, which the reference's
// unstable sort leaves open, go to the lower index here. This file computes the same rows without the
// O(n^2) triple list:
//
//   * knn_simt_kernel: every distance in the reference's exact f32 order (distance.rs:50-75) on CUDA
//     cores, each block keeping the running k' best (distance key, index) of 32 query rows in shared
//     memory. Used for small n, for any d, and as the fallback for rows the tensor-core filter
//     (knn_tc.cu) cannot settle. When there are too few query rows to fill the GPU, the keys are split
//     into slices (grid y); each slice writes its own k' best per row and knn_merge_kernel merges
//     them (the keys are totally ordered, so the merged lists are the same).
#include "engine.cuh"
#include "knn_tc.cuh"

namespace pacmap {
namespace {

constexpr int SQ_QB = 32;   // query rows per block
constexpr int SQ_KT = 64;   // keys per tile
constexpr int SQ_DC = 64;   // dimensions staged per pass (multiple of 8)
constexpr int SQ_LD = SQ_DC + 4;  // smem row stride (floats): 16-byte aligned, conflict-free float4 rows
constexpr int SQ_THREADS = 256;
constexpr int SQ_MAX_K = 448;     // P = next_pow2(K + KT) <= 512

__global__ void __launch_bounds__(SQ_THREADS) knn_simt_kernel(const float* __restrict__ x, uint64_t n, int d, int K,
                                                              int P, const uint32_t* __restrict__ rows,
                                                              uint64_t n_rows, uint32_t* __restrict__ out_idx,
                                                              float* __restrict__ out_dist, int scatter,
                                                              uint64_t slice, uint64_t* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* qs = reinterpret_cast<float*>(smem);
  float* ks = qs + SQ_QB * SQ_LD;
  uint64_t* lists = reinterpret_cast<uint64_t*>(ks + SQ_KT * SQ_LD);
  __shared__ int stage_cnt[SQ_QB];
  __shared__ uint64_t theta[SQ_QB];
  __shared__ uint64_t qrow[SQ_QB];

  const int tid = threadIdx.x;
  const int kt = tid & (SQ_KT - 1);
  const int qg = tid >> 6;  // 4 groups x 8 queries
  const uint64_t slot0 = static_cast<uint64_t>(blockIdx.x) * SQ_QB;

  if (tid < SQ_QB) {
    stage_cnt[tid] = 0;
    theta[tid] = ~0ull;
    const uint64_t s = slot0 + tid;
    qrow[tid] = (s < n_rows) ? (rows ? static_cast<uint64_t>(rows[s]) : s) : ~0ull;
  }
  for (int e = tid; e < SQ_QB * P; e += SQ_THREADS) lists[e] = ~0ull;
  __syncthreads();

  const int nc8 = (d / 8) * 8;  // the lane-accumulated part; the tail d % 8 is added after the lane sum
  // rows staged in 16-byte pieces when every row starts on a 16-byte boundary
  const bool vec4 = (d % 4 == 0) && ((reinterpret_cast<uintptr_t>(x) & 15u) == 0);
  // keys [kbeg, kend) of this block's slice (slice is a multiple of SQ_KT)
  const uint64_t kbeg = static_cast<uint64_t>(blockIdx.y) * slice;
  const uint64_t kend = kbeg + slice < n ? kbeg + slice : n;
  for (uint64_t key0 = kbeg; key0 < kend; key0 += SQ_KT) {
    float acc[8][8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
#pragma unroll
      for (int l = 0; l < 8; ++l) acc[q][l] = 0.0f;

    for (int dbase = 0; dbase < nc8; dbase += SQ_DC) {
      const int dlen = min(SQ_DC, nc8 - dbase);
      __syncthreads();
      if (vec4) {
        // 16-byte pieces, SQ_DC / 4 per row slot (pieces beyond this pass's dlen are skipped)
        const int q4 = dlen >> 2;
        for (int e = tid; e < SQ_QB * (SQ_DC / 4); e += SQ_THREADS) {
          const int qi = e / (SQ_DC / 4), c4 = e % (SQ_DC / 4);
          if (c4 >= q4) continue;
          const uint64_t r = qrow[qi];
          const float4 v = (r != ~0ull) ? *reinterpret_cast<const float4*>(x + r * d + dbase + 4 * c4)
                                        : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          *reinterpret_cast<float4*>(&qs[qi * SQ_LD + 4 * c4]) = v;
        }
        for (int e = tid; e < SQ_KT * (SQ_DC / 4); e += SQ_THREADS) {
          const int kk = e / (SQ_DC / 4), c4 = e % (SQ_DC / 4);
          if (c4 >= q4) continue;
          const uint64_t j = key0 + kk;
          const float4 v = (j < kend) ? *reinterpret_cast<const float4*>(x + j * d + dbase + 4 * c4)
                                      : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          *reinterpret_cast<float4*>(&ks[kk * SQ_LD + 4 * c4]) = v;
        }
      } else {
        for (int e = tid; e < SQ_QB * dlen; e += SQ_THREADS) {
          const int qi = e / dlen, cc = e - qi * dlen;
          const uint64_t r = qrow[qi];
          qs[qi * SQ_LD + cc] = (r != ~0ull) ? x[r * d + dbase + cc] : 0.0f;
        }
        for (int e = tid; e < SQ_KT * dlen; e += SQ_THREADS) {
          const int kk = e / dlen, cc = e - kk * dlen;
          const uint64_t j = key0 + kk;
          ks[kk * SQ_LD + cc] = (j < kend) ? x[j * d + dbase + cc] : 0.0f;
        }
      }
      __syncthreads();
      for (int c8 = 0; c8 < dlen; c8 += 8) {
        const float4 k0 = *reinterpret_cast<const float4*>(&ks[kt * SQ_LD + c8]);
        const float4 k1 = *reinterpret_cast<const float4*>(&ks[kt * SQ_LD + c8 + 4]);
        const float kv[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float* qp = &qs[(qg * 8 + q) * SQ_LD + c8];
          const float4 q0 = *reinterpret_cast<const float4*>(qp);
          const float4 q1 = *reinterpret_cast<const float4*>(qp + 4);
          const float qv[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
          for (int l = 0; l < 8; ++l) {
            const float df = __fsub_rn(qv[l], kv[l]);
            acc[q][l] = __fadd_rn(acc[q][l], __fmul_rn(df, df));
          }
        }
      }
    }

    const uint64_t j = key0 + kt;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int qi = qg * 8 + q;
      const uint64_t r = qrow[qi];
      float t = 0.0f;
#pragma unroll
      for (int l = 0; l < 8; ++l) t = __fadd_rn(t, acc[q][l]);
      if (r == ~0ull || j >= kend || j == r) continue;
      for (int e = nc8; e < d; ++e) {
        const float df = __fsub_rn(x[r * d + e], x[j * d + e]);
        t = __fadd_rn(t, __fmul_rn(df, df));
      }
      const float dist = __fsqrt_rn(t);
      const uint64_t key = (static_cast<uint64_t>(total_key(dist)) << 32) | j;
      if (key < theta[qi]) {
        const int pos = atomicAdd(&stage_cnt[qi], 1);
        lists[qi * P + K + pos] = key;
      }
    }
    __syncthreads();
    // Merge the staged candidates of each query into its sorted list (one warp per query).
    const int warp = tid >> 5, lane = tid & 31;
    for (int qi = warp; qi < SQ_QB; qi += SQ_THREADS / 32) {
      const int cnt = stage_cnt[qi];
      if (cnt == 0) continue;
      uint64_t* L = lists + qi * P;
      for (int e = K + cnt + lane; e < P; e += 32) L[e] = ~0ull;
      warp_bitonic_sort_u64(L, P);
      if (lane == 0) {
        stage_cnt[qi] = 0;
        theta[qi] = L[K - 1];
      }
      __syncwarp();
    }
    __syncthreads();
  }

  for (int e = tid; e < SQ_QB * K; e += SQ_THREADS) {
    const int qi = e / K, cc = e - qi * K;
    const uint64_t s = slot0 + qi;
    if (s >= n_rows) continue;
    const uint64_t key = lists[qi * P + cc];
    if (part) {  // one slice of several: its sorted k' best, merged by knn_merge_kernel
      part[(s * gridDim.y + blockIdx.y) * K + cc] = key;
      continue;
    }
    const uint64_t o = scatter ? qrow[qi] : s;
    out_idx[o * K + cc] = static_cast<uint32_t>(key & 0xFFFFFFFFu);
    out_dist[o * K + cc] = key_to_float(static_cast<uint32_t>(key >> 32));
  }
}

// One warp per query row: merges the rows' `slices` sorted lists of K keys into the K smallest, by
// repeated bitonic sorts of (running K best + next slice) in shared memory.
constexpr int MG_WARPS = 4;
__global__ void __launch_bounds__(MG_WARPS * 32) knn_merge_kernel(const uint64_t* __restrict__ part, int slices,
                                                                   int K, int P2, const uint32_t* __restrict__ rows,
                                                                   uint64_t n_rows, uint32_t* __restrict__ out_idx,
                                                                   float* __restrict__ out_dist, int scatter) {
  extern __shared__ __align__(16) unsigned char msmem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* buf = reinterpret_cast<uint64_t*>(msmem) + static_cast<size_t>(warp) * P2;
  const uint64_t s = static_cast<uint64_t>(blockIdx.x) * MG_WARPS + warp;
  if (s >= n_rows) return;
  const uint64_t* src = part + s * static_cast<uint64_t>(slices) * K;
  for (int e = lane; e < K; e += 32) buf[e] = src[e];
  for (int q = 1; q < slices; ++q) {
    __syncwarp();
    for (int e = lane; e < K; e += 32) buf[K + e] = src[static_cast<uint64_t>(q) * K + e];
    for (int e = 2 * K + lane; e < P2; e += 32) buf[e] = ~0ull;
    warp_bitonic_sort_u64(buf, P2);
  }
  __syncwarp();
  const uint64_t o = scatter ? static_cast<uint64_t>(rows[s]) : s;
  for (int e = lane; e < K; e += 32) {
    const uint64_t key = buf[e];
    out_idx[o * K + e] = static_cast<uint32_t>(key & 0xFFFFFFFFu);
    out_dist[o * K + e] = key_to_float(static_cast<uint32_t>(key >> 32));
  }
}

}  // namespace

void knn_rows_simt(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, const uint32_t* d_rows,
                   uint64_t n_rows, uint32_t* d_idx, float* d_dist, bool scatter) {
  if (n_rows == 0 || kp == 0) return;
  PM_REQUIRE(kp <= SQ_MAX_K, PACMAP_ERR_UNSUPPORTED,
             "exact kNN supports at most " + std::to_string(SQ_MAX_K) + " neighbours per row");
  PM_REQUIRE(n < (1ull << 32) && d < (1ull << 31), PACMAP_ERR_UNSUPPORTED, "kNN needs n < 2^32 and d < 2^31");
  const int K = static_cast<int>(kp);
  const int P = next_pow2(K + SQ_KT);
  const size_t smem = static_cast<size_t>(SQ_QB + SQ_KT) * SQ_LD * sizeof(float) + static_cast<size_t>(SQ_QB) * P * 8;
  PM_CUDA(cudaFuncSetAttribute(knn_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  // Key slices: enough blocks for two waves when the query rows alone do not fill the GPU; every slice
  // keeps at least 4096 keys (a multiple of the key tile).
  int per_sm = 1;
  PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, knn_simt_kernel, SQ_THREADS, smem));
  const uint64_t row_blocks = ceil_div(n_rows, SQ_QB);
  const uint64_t want = 2ull * c.sm_count * static_cast<uint64_t>(std::max(per_sm, 1));
  uint64_t slices = std::min<uint64_t>((want + row_blocks - 1) / row_blocks, std::max<uint64_t>(n / 4096, 1));
  slices = std::min<uint64_t>(slices, 1024);
  slices = std::max<uint64_t>(slices, 1);
  uint64_t slice = (n + slices - 1) / slices;
  slice = (slice + SQ_KT - 1) / SQ_KT * SQ_KT;
  slices = (n + slice - 1) / slice;
  DevBuf<uint64_t> part;
  if (slices > 1) part.alloc(c, n_rows * slices * static_cast<uint64_t>(K));
  const dim3 grid(static_cast<unsigned>(row_blocks), static_cast<unsigned>(slices));
  knn_simt_kernel<<<grid, SQ_THREADS, smem, c.stream>>>(d_x, n, static_cast<int>(d), K, P, d_rows, n_rows, d_idx,
                                                         d_dist, scatter ? 1 : 0, slice,
                                                         slices > 1 ? part.get() : nullptr);
  PM_LAUNCHED();
  if (slices > 1) {
    const int P2 = next_pow2(2 * K);
    const size_t msm = static_cast<size_t>(MG_WARPS) * P2 * sizeof(uint64_t);
    PM_CUDA(cudaFuncSetAttribute(knn_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(msm)));
    knn_merge_kernel<<<ceil_div(n_rows, MG_WARPS), MG_WARPS * 32, msm, c.stream>>>(
        part.get(), static_cast<int>(slices), K, P2, d_rows, n_rows, d_idx, d_dist, scatter ? 1 : 0);
    PM_LAUNCHED();
  }
}

__global__ void iota_rows_kernel(uint32_t* __restrict__ rows, uint64_t r0, uint64_t count,
                                 uint8_t* __restrict__ owned) {
  const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= count) return;
  rows[t] = static_cast<uint32_t>(r0 + t);
  if (owned) owned[r0 + t] = 1;
}

void knn_exact_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, int mode, uint32_t* d_idx,
                      float* d_dist, const KnnShard& shard, uint64_t approx_threshold) {
  if (n == 0 || kp == 0) return;
  PM_REQUIRE(shard.count >= 1 && shard.index < shard.count, PACMAP_ERR_INVALID_ARGUMENT, "bad kNN shard");
  // AUTO uses the tensor cores once the O(n^2) part dominates; the TENSOR modes force them.
  const bool approx = mode == PACMAP_KNN_APPROX && n >= approx_threshold;
  const bool want_tc = (mode == PACMAP_KNN_TENSOR_F16 || mode == PACMAP_KNN_TENSOR_BF16 ||
                        mode == PACMAP_KNN_TENSOR_F16_FULL) ||
                       ((mode == PACMAP_KNN_AUTO || mode == PACMAP_KNN_APPROX) && n >= 16384);
  if (want_tc && knn_tc_supported(n, d, kp)) {
    if (knn_tc_device(c, d_x, n, d, kp, mode == PACMAP_KNN_TENSOR_BF16, d_idx, d_dist, shard, approx ? 16 : 0,
                      /*prune=*/mode != PACMAP_KNN_TENSOR_F16_FULL))
      return;
  }
  PM_REQUIRE(mode == PACMAP_KNN_AUTO || mode == PACMAP_KNN_SIMT_EXACT || mode == PACMAP_KNN_APPROX,
             PACMAP_ERR_UNSUPPORTED,
             "the tensor-core kNN does not support this shape (d <= 1024 and k' <= 447 are required)");
  if (shard.count == 1) {
    knn_rows_simt(c, d_x, n, d, kp, nullptr, n, d_idx, d_dist);
    if (shard.d_owned) PM_CUDA(cudaMemsetAsync(shard.d_owned, 1, n, c.stream));
    return;
  }
  const uint64_t r0 = n * shard.index / shard.count, r1 = n * (shard.index + 1) / shard.count;
  if (r1 == r0) return;
  DevBuf<uint32_t> rows(c, r1 - r0);
  iota_rows_kernel<<<ceil_div(r1 - r0, 256), 256, 0, c.stream>>>(rows.get(), r0, r1 - r0, shard.d_owned);
  PM_LAUNCHED();
  knn_rows_simt(c, d_x, n, d, kp, rows.get(), r1 - r0, d_idx, d_dist, /*scatter=*/true);
}

}  // namespace pacmap
