// Pivots of the locality order, and certified tile pruning for the exact tensor-core kNN.
//
// The filter (knn_tc.cu) runs the distance GEMM of every (row block of 256, column tile of 128) pair of
// the locality order. Most pairs cannot hold a neighbour. Through any pivot p the triangle inequality
// bounds a distance from below, |x_i - x_j| >= | |x_i - p| - |x_j - p| |, so for a row segment s and a
// column segment t (the rows of one pivot cell inside one tile):
//     min over i in s, j in t of |x_i - x_j|  >=  LB(s, t) = max( m_s(p_t) - R_t, m_t(p_s) - R_s ),
// with p_s the pivot of s's cell, R_s = max_{i in s} |x_i - p_s| (the segment's radius) and
// m_s(p) = min_{i in s} |x_i - p|. A first filter pass over the cells nearest each block gives every
// row i an upper bound U_i of its k'-th neighbour distance (any k' other points give one). A column tile
// is skipped for a row block when LB(s, t) > max_{i in s} U_i for every row segment s of the block and
// every segment t of the tile: no point of the tile can be among the k' nearest of any of the block's
// rows, ties included. The kept tiles go through the unchanged filter, whose candidate sets stay
// complete, so the exact re-rank returns the reference's rows (src/knn.rs:137-194) bit for bit.
// Every bound is widened for its f32 rounding: the pivot distances by an explicit error term, and the
// final comparison by a relative margin of 1e-4 that also covers the reference's own f32 distance sum.
//
// Pivots: k-means++ seeding (Arthur & Vassilvitskii, SODA 2007) in batches of 16 draws on a subsample of
// at most 65,536 rows, so that every well-separated group of points receives a pivot and the cells stay
// compact; the draws come from a Philox4x32-10 stream with a fixed key (the same pivots on every call).
#include <algorithm>
#include <cmath>

#include "knn_layout.cuh"
#include "knn_prune.cuh"

namespace pacmap {

namespace {

constexpr int PV_BATCH = 16;             // pivots drawn per round
constexpr uint32_t PV_SUB_MAX = 65536;   // subsample size limit
constexpr int PV_CHUNK = 256;            // subsample points per block (and per prefix-sum entry)
constexpr uint32_t TAG_PIVOT = 0x50495654u;  // 'PIVT'
constexpr int SEGS = 4;                  // cell segments kept per tile (further cells merge into the last)
constexpr float PRUNE_MARGIN = 1e-4f;    // relative margin of the skip test

__host__ __device__ __forceinline__ uint64_t sub_row(uint32_t s, uint32_t S, uint64_t n) {
  return static_cast<uint64_t>(s) * n / S;
}

// dmin[s] = min(dmin[s], |x_row(s) - q|^2 over the 16 pivots q of the batch starting at p0) for the
// subsample points of this block's chunk, and the chunk's sum of dmin (f64, a fixed order). p0 == 0
// starts dmin from +inf. One warp per point, lanes over the columns; the batch is staged in shared memory.
__global__ void __launch_bounds__(256) pivot_dmin_kernel(const float* __restrict__ x, uint64_t n, int d, uint32_t S,
                                                         const uint32_t* __restrict__ piv_rows, int p0,
                                                         float* __restrict__ dmin, double* __restrict__ chunk_sum) {
  extern __shared__ float pv[];  // PV_BATCH x d
  __shared__ double wsum[8];
  for (int e = threadIdx.x; e < PV_BATCH * d; e += blockDim.x) {
    const int q = e / d, col = e - q * d;
    pv[e] = x[static_cast<uint64_t>(piv_rows[p0 + q]) * d + col];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int PER_WARP = PV_CHUNK / 8;
  double ws = 0.0;
  // four subsample rows at a time (their loads in flight together); each row's sums and the order of
  // the block's double sum are those of one row at a time
  static_assert(PER_WARP % 4 == 0, "rows are taken four at a time");
  for (int t0 = 0; t0 < PER_WARP; t0 += 4) {
    const uint32_t s0 = blockIdx.x * PV_CHUNK + warp * PER_WARP + t0;
    if (s0 >= S) break;  // warp-uniform
    const float* xr[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xr[u] = x + sub_row(s0 + u < S ? s0 + u : s0, S, n) * d;
    float acc[4][PV_BATCH];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int q = 0; q < PV_BATCH; ++q) acc[u][q] = 0.0f;
    for (int col = lane; col < d; col += 32) {
      float xv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) xv[u] = xr[u][col];
#pragma unroll
      for (int q = 0; q < PV_BATCH; ++q) {
        const float pq = pv[q * d + col];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float df = xv[u] - pq;
          acc[u][q] = fmaf(df, df, acc[u][q]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t s = s0 + u;
      if (s >= S) break;  // warp-uniform
      float best = p0 == 0 ? __int_as_float(0x7f800000) : dmin[s];
#pragma unroll
      for (int q = 0; q < PV_BATCH; ++q) {
        float v = acc[u][q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);  // the same sum on every lane
        best = fminf(best, v);
      }
      if (lane == 0) dmin[s] = best;
      if (best < 3.0e38f) ws += static_cast<double>(best);
    }
  }
  if (lane == 0) wsum[warp] = ws;
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int w = 0; w < 8; ++w) total += wsum[w];
    chunk_sum[blockIdx.x] = total;
  }
}

// Round 0: 16 evenly spaced subsample points. Round r > 0: 16 draws, each point with probability
// proportional to dmin (its squared distance to the nearest pivot so far); a degenerate subsample (all
// dmin zero) falls back to evenly spaced points.
__global__ void __launch_bounds__(PV_BATCH * 32) pivot_draw_kernel(const float* __restrict__ dmin, uint32_t S,
                                                                   uint64_t n, const double* __restrict__ chunk_sum,
                                                                   int nchunks, int round,
                                                                   uint32_t* __restrict__ piv_rows) {
  __shared__ double cs[PV_SUB_MAX / PV_CHUNK];
  __shared__ double pre[PV_SUB_MAX / PV_CHUNK + 1];
  for (int ch = threadIdx.x; round > 0 && ch < nchunks; ch += blockDim.x) cs[ch] = chunk_sum[ch];
  __syncthreads();
  if (threadIdx.x == 0) {  // the prefix in chunk order, from shared memory
    double run = 0.0;
    pre[0] = 0.0;
    for (int ch = 0; round > 0 && ch < nchunks; ++ch) {
      const double v = cs[ch];
      run += (v > 0.0 && v < 1e300) ? v : 0.0;
      pre[ch + 1] = run;
    }
  }
  __syncthreads();
  // one warp per draw: the chunk's dmin values read 32 at a time, then added in index order on every lane
  // (the same sequence of double additions as one thread walking the chunk)
  const int b = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
  uint32_t s = round == 0 ? static_cast<uint32_t>(static_cast<uint64_t>(b) * S / PV_BATCH)
                          : static_cast<uint32_t>(static_cast<uint64_t>(round * PV_BATCH + b) * S / PIV);
  const double total = round > 0 ? pre[nchunks] : 0.0;
  if (round > 0 && total > 0.0 && total < 1e300) {
    uint32_t w[4];
    philox4x32_10(static_cast<uint32_t>(round), static_cast<uint32_t>(b), 0u, TAG_PIVOT, 0x9E3779B9u, 0x7F4A7C15u, w);
    const uint64_t bits53 = (static_cast<uint64_t>(w[0]) << 21) | (w[1] >> 11);
    const double target = static_cast<double>(bits53) * (1.0 / 9007199254740992.0) * total;
    int lo = 0, hi = nchunks - 1;  // the last chunk whose prefix is <= target
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre[mid] <= target) lo = mid;
      else hi = mid - 1;
    }
    double acc = pre[lo];
    const uint32_t a = static_cast<uint32_t>(lo) * PV_CHUNK, e = min(S, a + PV_CHUNK);
    uint32_t pick = 0xFFFFFFFFu;
    bool done = false;
    for (uint32_t base = a; base < e && !done; base += 32) {
      const uint32_t t = base + static_cast<uint32_t>(lane);
      const float mine = t < e ? dmin[t] : 0.0f;
      for (int k = 0; k < 32; ++k) {
        const float v = __shfl_sync(0xFFFFFFFFu, mine, k);
        if (!done && base + k < e && v > 0.0f && v < 3.0e38f) {
          pick = base + static_cast<uint32_t>(k);
          acc += v;
          if (acc > target) done = true;
        }
      }
    }
    if (pick != 0xFFFFFFFFu) s = pick;
  }
  if (lane == 0) piv_rows[round * PV_BATCH + b] = static_cast<uint32_t>(sub_row(s, S, n));
}

// Per column tile (128 positions): its rows split by pivot cell into at most SEGS segments (cells are
// contiguous in the locality order; cells past the fourth merge into the fourth, whose pivot stays its
// first cell's). Per segment g: seg_cell, the radius seg_rad = max |x_i - p_cell| (rounded up), the
// largest row bound seg_ub = max U_i, and for every pivot p, minT[p * nseg + g] = min |x_i - p| (rounded
// down). One thread per pivot; a non-finite distance or bound makes the segment unprunable (-inf / +inf).
__global__ void __launch_bounds__(PIV) seg_stats_kernel(PruneInputs in, float errc, int* __restrict__ seg_cell,
                                                        float* __restrict__ seg_rad, float* __restrict__ seg_ub,
                                                        float* __restrict__ minT, uint64_t nseg) {
  __shared__ float rad_s[SEGS];
  const uint64_t tile = blockIdx.x;
  const uint64_t r0 = tile * TC_BN, r1 = min(r0 + TC_BN, in.n);
  const int p = threadIdx.x;
  const float inf = __int_as_float(0x7f800000);
  const float inv_s2 = in.inv_s * in.inv_s;
  float mn[SEGS], rad[SEGS], ubm[SEGS];
  int cl[SEGS];
#pragma unroll
  for (int q = 0; q < SEGS; ++q) {
    mn[q] = inf;
    rad[q] = 0.0f;
    ubm[q] = 0.0f;
    cl[q] = -1;
  }
  const float pn = in.pnorm[p];
  int s = -1;
  uint32_t prev = 0xFFFFFFFFu;
  for (uint64_t r = r0; r < r1; ++r) {
    const uint32_t o = in.perm[r];
    const uint32_t cc = in.cell[o];
    if (cc != prev) {
      prev = cc;
      if (s < SEGS - 1) {
        ++s;
#pragma unroll
        for (int q = 0; q < SEGS; ++q)
          if (q == s) cl[q] = static_cast<int>(cc);
      }
    }
    const float xn = in.rownorm[r] * inv_s2;  // |x|^2: the scale is an exact power of two
    const float d2 = in.score[static_cast<uint64_t>(o) * PIV + p] + xn;
    const float err = errc * (xn + pn);
    float lo = sqrtf(fmaxf(d2 - err, 0.0f)) * (1.0f - 2.4e-7f);
    if (!(lo >= 0.0f)) lo = -inf;  // NaN
    float hi = sqrtf(d2 + err) * (1.0f + 2.4e-7f);
    if (!(hi <= 3.4e38f)) hi = inf;
    float u = 0.0f;
    if (p == 0) {
      const float ub = in.ub[r];
      u = ub >= 0.0f ? sqrtf(ub) * in.inv_s * (1.0f + 4.8e-7f) : inf;
      if (!(u <= 3.4e38f)) u = inf;
    }
#pragma unroll
    for (int q = 0; q < SEGS; ++q) {
      if (q == s) {
        mn[q] = fminf(mn[q], lo);
        if (p == cl[q]) rad[q] = fmaxf(rad[q], hi);
        if (p == 0) ubm[q] = fmaxf(ubm[q], u);
      }
    }
  }
  // each segment's radius lives in the thread of its pivot
#pragma unroll
  for (int q = 0; q < SEGS; ++q)
    if (cl[q] == p) rad_s[q] = rad[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < SEGS; ++q) minT[static_cast<uint64_t>(p) * nseg + tile * SEGS + q] = mn[q];
  if (p == 0) {
#pragma unroll
    for (int q = 0; q < SEGS; ++q) {
      seg_cell[tile * SEGS + q] = cl[q];
      seg_rad[tile * SEGS + q] = cl[q] >= 0 ? rad_s[q] : 0.0f;
      seg_ub[tile * SEGS + q] = ubm[q];
    }
  }
}

// One block per row block: the visit bit of every column tile and the count of visited tiles. The
// block's row segments are those of its two tiles; a tile is visited unless every (row segment, tile
// segment) pair is separated by more than the row segment's bound. The block's own tiles are always kept.
__global__ void __launch_bounds__(256) prune_tiles_kernel(const int* __restrict__ seg_cell,
                                                          const float* __restrict__ seg_rad,
                                                          const float* __restrict__ seg_ub,
                                                          const float* __restrict__ minT, uint64_t nseg, int ntiles,
                                                          int words, int blk0, const uint32_t* __restrict__ skip_ptr,
                                                          const uint32_t* __restrict__ skip_list,
                                                          uint32_t* __restrict__ bits, uint32_t* __restrict__ counts) {
  __shared__ float ms[2 * SEGS][PIV];
  __shared__ int sp[2 * SEGS];
  __shared__ float srad[2 * SEGS], sthr[2 * SEGS];
  __shared__ uint32_t wcount[8];
  const int blk = static_cast<int>(blockIdx.x) + blk0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint64_t g0 = static_cast<uint64_t>(2 * blk) * SEGS;
  if (tid < 2 * SEGS) {
    const int cl = seg_cell[g0 + tid];
    sp[tid] = cl;
    srad[tid] = cl >= 0 ? seg_rad[g0 + tid] : 0.0f;
    sthr[tid] = cl >= 0 ? seg_ub[g0 + tid] * (1.0f + PRUNE_MARGIN) : 0.0f;
  }
  __syncthreads();
  for (int q = 0; q < 2 * SEGS; ++q) ms[q][tid] = sp[q] >= 0 ? minT[static_cast<uint64_t>(tid) * nseg + g0 + q] : 0.0f;
  __syncthreads();
  uint32_t cnt = 0;
  for (int base = 0; base < ntiles; base += 256) {
    const int J = base + tid;
    bool visit = false;
    if (J < ntiles) {
      visit = (J >> 1) == blk;
      for (int qt = 0; qt < SEGS && !visit; ++qt) {
        const uint64_t t = static_cast<uint64_t>(J) * SEGS + qt;
        const int pt = seg_cell[t];
        if (pt < 0) break;  // segments are filled in order
        const float rt = seg_rad[t];
        for (int qs = 0; qs < 2 * SEGS; ++qs) {
          const int ps = sp[qs];
          if (ps < 0) continue;
          const float lb = fmaxf(ms[qs][pt] - rt, minT[static_cast<uint64_t>(ps) * nseg + t] - srad[qs]);
          if (!(lb * (1.0f - PRUNE_MARGIN) > sthr[qs])) {
            visit = true;
            break;
          }
        }
      }
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, visit);
    const int word = (base >> 5) + warp;
    if (lane == 0 && word < words) bits[static_cast<uint64_t>(blk) * words + word] = bal;
  }
  uint32_t* mine = bits + static_cast<uint64_t>(blk) * words;
  if (skip_ptr) {
    __syncthreads();
    for (uint32_t e = skip_ptr[blk] + tid; e < skip_ptr[blk + 1]; e += blockDim.x) {
      const uint32_t t = skip_list[e];
      atomicAnd(&mine[t >> 5], ~(1u << (t & 31)));
    }
    __syncthreads();
  }
  for (int w = tid; w < words; w += blockDim.x) cnt += __popc(mine[w]);
  cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
  if (lane == 0) wcount[warp] = cnt;
  __syncthreads();
  if (tid == 0) {
    uint32_t total = 0;
    for (int w = 0; w < 8; ++w) total += wcount[w];
    counts[blk] = total;
  }
}

// ptr[b] = sum of counts[0..b), ptr[nb] the total (one block).
__global__ void __launch_bounds__(1024) scan_counts_kernel(const uint32_t* __restrict__ counts, uint64_t nb,
                                                           uint32_t* __restrict__ ptr) {
  __shared__ uint32_t part[1024];
  const uint64_t per = (nb + 1023) / 1024;
  const uint64_t a = threadIdx.x * per, e = min(nb, a + per);
  uint32_t s = 0;
  for (uint64_t i = a; i < e; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const uint32_t v = threadIdx.x >= static_cast<unsigned>(o) ? part[threadIdx.x - o] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
  for (uint64_t i = a; i < e; ++i) {
    ptr[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == 1023) ptr[nb] = part[1023];
}

// One warp per row block: its visited tiles in the sweep order (the window around its own rows first).
__global__ void __launch_bounds__(128) fill_tile_lists_kernel(const uint32_t* __restrict__ bits, int words, int ntiles,
                                                              const uint32_t* __restrict__ ptr, int blk0, int nblk,
                                                              uint32_t* __restrict__ list) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = static_cast<int>(blockIdx.x) * 4 + warp;
  if (j >= nblk) return;
  const int blk = blk0 + j;
  uint32_t pos = ptr[blk];
  for (int t0 = 0; t0 < ntiles; t0 += 32) {
    const int t = t0 + lane;
    bool v = false;
    int tile = 0;
    if (t < ntiles) {
      tile = sweep_tile(t, blk, ntiles);
      v = (bits[static_cast<uint64_t>(blk) * words + (tile >> 5)] >> (tile & 31)) & 1u;
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, v);
    if (v) list[pos + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint32_t>(tile);
    pos += __popc(bal);
  }
}

// near[p * probe + r]: the `probe` pivots nearest pivot p, itself first, by f32 squared distance of the
// pivot rows, ties to the lower index. One block per pivot, one thread per other pivot.
__global__ void __launch_bounds__(PIV) pivot_near_kernel(const float* __restrict__ x,
                                                         const uint32_t* __restrict__ piv_rows, int d, int probe,
                                                         uint32_t* __restrict__ near) {
  __shared__ uint64_t best[PIV / 32];
  const int p = blockIdx.x, q = threadIdx.x, warp = q >> 5, lane = q & 31;
  const float* xp = x + static_cast<uint64_t>(piv_rows[p]) * d;
  const float* xq = x + static_cast<uint64_t>(piv_rows[q]) * d;
  float acc = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float df = xp[k] - xq[k];
    acc = fmaf(df, df, acc);
  }
  uint64_t key = q == p ? 0ull : ((static_cast<uint64_t>(total_key(acc)) << 32) | static_cast<uint32_t>(q));
  for (int r = 0; r < probe; ++r) {
    uint64_t m = key;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t t = __shfl_xor_sync(0xFFFFFFFFu, m, o);
      m = t < m ? t : m;
    }
    if (lane == 0) best[warp] = m;
    __syncthreads();
    uint64_t b = best[0];
    for (int w = 1; w < PIV / 32; ++w) b = best[w] < b ? best[w] : b;
    const int winner = b == 0ull ? p : static_cast<int>(b & 0xFFFFFFFFu);
    if (q == 0) near[p * probe + r] = static_cast<uint32_t>(winner);
    if (q == winner) key = ~0ull;
    __syncthreads();
  }
}

// Per row block: the column tiles of its own cells, then those of the probe - 1 cells nearest each of its
// own cells that holds fewer than min_cell points (ascending tile order in each group, no repeats). Count
// pass (list == nullptr) or fill pass.
constexpr int PL_MAX_WORDS = 4096;  // tile bitmask words in shared memory (ntiles <= 131,072)
__global__ void __launch_bounds__(PIV) probe_lists_kernel(const uint32_t* __restrict__ cstart, uint64_t n, int ntiles,
                                                          const uint32_t* __restrict__ near, int probe,
                                                          uint32_t min_cell, int blk0,
                                                          const uint32_t* __restrict__ ptr,
                                                          uint32_t* __restrict__ counts, uint32_t* __restrict__ list) {
  __shared__ uint32_t own[PL_MAX_WORDS], other[PL_MAX_WORDS];
  __shared__ uint32_t wsum[PIV / 32];
  const int words = (ntiles + 31) / 32;
  const int b = static_cast<int>(blockIdx.x) + blk0, p = threadIdx.x;
  for (int w = p; w < words; w += PIV) own[w] = other[w] = 0u;
  __syncthreads();
  const uint64_t r0 = static_cast<uint64_t>(b) * TC_BM, r1 = min(r0 + TC_BM, n);
  auto mark = [&](uint32_t* mask, int q) {
    const uint32_t a = cstart[q], e = q + 1 < PIV ? cstart[q + 1] : static_cast<uint32_t>(n);
    if (e <= a) return;
    for (uint32_t t = a / TC_BN; t <= (e - 1) / TC_BN; ++t) atomicOr(&mask[t >> 5], 1u << (t & 31));
  };
  const uint32_t a = cstart[p], e = p + 1 < PIV ? cstart[p + 1] : static_cast<uint32_t>(n);
  const bool mine = r0 < r1 && a < r1 && e > r0;
  if (mine) mark(own, p);
  __syncthreads();
  if (mine && e - a < min_cell)
    for (int r = 1; r < probe; ++r) mark(other, static_cast<int>(near[p * probe + r]));
  __syncthreads();
  uint32_t c = 0;
  for (int w = p; w < words; w += PIV) {
    other[w] &= ~own[w];
    c += __popc(own[w]) + __popc(other[w]);
  }
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  if ((p & 31) == 0) wsum[p >> 5] = c;
  __syncthreads();
  if (!list) {
    if (p == 0) {
      uint32_t t = 0;
      for (int w = 0; w < PIV / 32; ++w) t += wsum[w];
      counts[b] = t;
    }
    return;
  }
  if (p == 0) {
    uint32_t pos = ptr[b];
    for (int g = 0; g < 2; ++g) {
      const uint32_t* mask = g == 0 ? own : other;
      for (int w = 0; w < words; ++w)
        for (uint32_t m = mask[w]; m; m &= m - 1) list[pos++] = static_cast<uint32_t>(w * 32 + __ffs(m) - 1);
    }
  }
}

}  // namespace

uint64_t build_probe_tile_lists(Ctx& c, const float* d_x, uint64_t d, const uint32_t* d_piv_rows,
                                const uint32_t* d_cstart, uint64_t n, uint64_t n_pad, int probe, uint32_t min_cell,
                                uint64_t blk0, uint64_t blk1, DevBuf<uint32_t>& ptr, DevBuf<uint32_t>& list) {
  const uint64_t nb = n_pad / TC_BM, ntiles = n_pad / TC_BN;
  PM_REQUIRE((ntiles + 31) / 32 <= static_cast<uint64_t>(PL_MAX_WORDS) && probe >= 1 && probe <= PIV,
             PACMAP_ERR_UNSUPPORTED, "probe lists: too many tiles");
  DevBuf<uint32_t> near(c, static_cast<uint64_t>(PIV) * probe), counts(c, nb);
  pivot_near_kernel<<<PIV, PIV, 0, c.stream>>>(d_x, d_piv_rows, static_cast<int>(d), probe, near.get());
  PM_LAUNCHED();
  PM_CUDA(cudaMemsetAsync(counts.get(), 0, nb * sizeof(uint32_t), c.stream));
  const unsigned nblk = static_cast<unsigned>(blk1 - blk0);
  if (nblk) {
    probe_lists_kernel<<<nblk, PIV, 0, c.stream>>>(d_cstart, n, static_cast<int>(ntiles), near.get(), probe, min_cell,
                                                   static_cast<int>(blk0), nullptr, counts.get(), nullptr);
    PM_LAUNCHED();
  }
  ptr.alloc(c, nb + 1);
  scan_counts_kernel<<<1, 1024, 0, c.stream>>>(counts.get(), nb, ptr.get());
  PM_LAUNCHED();
  uint32_t total = 0;
  PM_CUDA(cudaMemcpyAsync(&total, ptr.get() + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  list.alloc(c, std::max<uint64_t>(total, 1));
  if (nblk) {
    probe_lists_kernel<<<nblk, PIV, 0, c.stream>>>(d_cstart, n, static_cast<int>(ntiles), near.get(), probe, min_cell,
                                                   static_cast<int>(blk0), ptr.get(), counts.get(), list.get());
    PM_LAUNCHED();
  }
  return total;
}

void select_pivots(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint32_t* d_piv_rows) {
  const uint32_t S = static_cast<uint32_t>(std::min<uint64_t>(n, PV_SUB_MAX));
  const int nchunks = static_cast<int>(ceil_div(S, PV_CHUNK));
  DevBuf<float> dmin(c, S);
  DevBuf<double> csum(c, nchunks);
  const size_t smem = static_cast<size_t>(PV_BATCH) * d * sizeof(float);
  PM_CUDA(cudaFuncSetAttribute(pivot_dmin_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  pivot_draw_kernel<<<1, PV_BATCH * 32, 0, c.stream>>>(dmin.get(), S, n, csum.get(), nchunks, 0, d_piv_rows);
  PM_LAUNCHED();
  for (int r = 1; r < PIV / PV_BATCH; ++r) {
    pivot_dmin_kernel<<<nchunks, 256, smem, c.stream>>>(d_x, n, static_cast<int>(d), S, d_piv_rows, (r - 1) * PV_BATCH,
                                                        dmin.get(), csum.get());
    PM_LAUNCHED();
    pivot_draw_kernel<<<1, PV_BATCH * 32, 0, c.stream>>>(dmin.get(), S, n, csum.get(), nchunks, r, d_piv_rows);
    PM_LAUNCHED();
  }
}

uint64_t build_pruned_tile_lists(Ctx& c, const PruneInputs& in, DevBuf<uint32_t>& ptr, DevBuf<uint32_t>& list) {
  const uint64_t nb = in.n_pad / TC_BM, ntiles = in.n_pad / TC_BN;
  const uint64_t nseg = ntiles * SEGS;
  const int words = static_cast<int>((ntiles + 31) / 32);
  DevBuf<int> seg_cell(c, nseg);
  DevBuf<float> seg_rad(c, nseg), seg_ub(c, nseg), minT(c, static_cast<uint64_t>(PIV) * nseg);
  // |p|^2 - 2 x.p + |x|^2 with fused multiply-add sums over d terms: within (3d + 16) 2^-24 (|x|^2 + |p|^2)
  const float errc = static_cast<float>(3 * in.d + 16) * 5.9604644775390625e-08f;
  seg_stats_kernel<<<static_cast<unsigned>(ntiles), PIV, 0, c.stream>>>(in, errc, seg_cell.get(), seg_rad.get(),
                                                                         seg_ub.get(), minT.get(), nseg);
  PM_LAUNCHED();
  DevBuf<uint32_t> bits(c, nb * words), counts(c, nb);
  PM_CUDA(cudaMemsetAsync(counts.get(), 0, nb * sizeof(uint32_t), c.stream));
  const unsigned nblk = static_cast<unsigned>(in.blk1 - in.blk0);
  if (nblk) {
    prune_tiles_kernel<<<nblk, 256, 0, c.stream>>>(seg_cell.get(), seg_rad.get(), seg_ub.get(), minT.get(), nseg,
                                                   static_cast<int>(ntiles), words, static_cast<int>(in.blk0),
                                                   in.skip_ptr, in.skip_list, bits.get(), counts.get());
    PM_LAUNCHED();
  }
  ptr.alloc(c, nb + 1);
  scan_counts_kernel<<<1, 1024, 0, c.stream>>>(counts.get(), nb, ptr.get());
  PM_LAUNCHED();
  uint32_t total = 0;
  PM_CUDA(cudaMemcpyAsync(&total, ptr.get() + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  list.alloc(c, std::max<uint64_t>(total, 1));
  if (nblk) {
    fill_tile_lists_kernel<<<ceil_div(nblk, 4), 128, 0, c.stream>>>(bits.get(), words, static_cast<int>(ntiles),
                                                                    ptr.get(), static_cast<int>(in.blk0),
                                                                    static_cast<int>(nblk), list.get());
    PM_LAUNCHED();
  }
  return total;
}

}  // namespace pacmap
