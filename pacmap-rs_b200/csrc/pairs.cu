// Pair generation after the kNN -- src/neighbors.rs:56-108 and src/sampling.rs:37-313.
//
//   K4 sigma_kernel / reselect_kernel: sigma_i = mean(dist[i, 3..6]) floored at 1e-10
//      (neighbors.rs:79-84), scaled = d*d / (sigma_i*sigma_j) (distance.rs:27-37), each row's k' scaled
//      distances ordered by f32::total_cmp (ties: lower kNN column) and the first k kept
//      (sampling.rs:251-286). One warp per row, bitonic sort in shared memory.
//   K5 sample_fp_kernel: far pairs (sampling.rs:37-103): n_fp distinct partners per point, not the
//      point, not among its k nearest neighbours, by rejection on the point's Philox stream.
//   K6 sample_mn_kernel: mid-near pairs (sampling.rs:118-142, 296-313): per slot, 6 distinct
//      candidates (not the point, not an earlier pick), the 2nd smallest reference f32 distance wins.
//
// Both samplers give one warp to one point. The fast variants draw from a WarpStream (each lane
// computes one Philox block per 128 words and the words are shuffled out) and keep the point's
// exclusion lists in registers (slot s in lane s % 32, register s / 32), so a membership test is one
// compare per register and a vote; the MN variant also keeps row i of x in registers. The general
// variants (every lane replays the stream, lists read from memory) serve the shapes beyond those
// registers. Both variants consume the same words in the same order: the pairs are identical.
#include <cuda_fp16.h>

#include <type_traits>

#include "engine.cuh"

namespace pacmap {
namespace {

__global__ void sigma_kernel(const float* __restrict__ kd, uint64_t n, int kp, float* __restrict__ sig) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int start = min(3, kp > 0 ? kp - 1 : 0);
  const int end = min(6, kp);
  if (end <= start) {
    sig[i] = 1e-10f;
    return;
  }
  float s = 0.0f;
  for (int cc = start; cc < end; ++cc) s = __fadd_rn(s, kd[i * kp + cc]);
  const float m = __fdiv_rn(s, static_cast<float>(end - start));
  sig[i] = fmaxf(m, 1e-10f);
}

constexpr int RS_WARPS = 4;

__global__ void __launch_bounds__(RS_WARPS * 32) reselect_kernel(const uint32_t* __restrict__ nbr,
                                                                 const float* __restrict__ kd,
                                                                 const float* __restrict__ sig, uint64_t n, int kp,
                                                                 int k, int P, uint32_t* __restrict__ pnn) {
  extern __shared__ uint64_t rs_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* buf = rs_smem + warp * P;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * RS_WARPS + warp; i < n;
       i += static_cast<uint64_t>(gridDim.x) * RS_WARPS) {
    const float si = sig[i];
    auto key_of = [&](int cc) -> uint64_t {
      if (cc >= kp) return ~0ull;
      const float dd = kd[i * kp + cc];
      const float s = __fdiv_rn(__fmul_rn(dd, dd), __fmul_rn(si, sig[nbr[i * kp + cc]]));
      return (static_cast<uint64_t>(total_key(s)) << 32) | static_cast<uint32_t>(cc);
    };
    if (P <= 128) {  // in registers: up to 4 keys per lane
      auto sort_regs = [&](auto tag) {
        constexpr int R = decltype(tag)::value;
        uint64_t v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = key_of(r * 32 + lane);
        warp_sort_regs_u64<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = r * 32 + lane;
          if (j < k) {
            const uint32_t cc = static_cast<uint32_t>(v[r] & 0xFFFFFFFFu);
            pnn[(i * k + j) * 2 + 0] = static_cast<uint32_t>(i);
            pnn[(i * k + j) * 2 + 1] = nbr[i * kp + cc];
          }
        }
      };
      if (P <= 32) sort_regs(std::integral_constant<int, 1>());
      else if (P <= 64) sort_regs(std::integral_constant<int, 2>());
      else sort_regs(std::integral_constant<int, 4>());
      continue;
    }
    for (int cc = lane; cc < P; cc += 32) buf[cc] = key_of(cc);
    warp_bitonic_sort_u64(buf, P);
    for (int j = lane; j < k; j += 32) {
      const uint32_t cc = static_cast<uint32_t>(buf[j] & 0xFFFFFFFFu);
      pnn[(i * k + j) * 2 + 0] = static_cast<uint32_t>(i);
      pnn[(i * k + j) * 2 + 1] = nbr[i * kp + cc];
    }
    __syncwarp();
  }
}

// True when any lane finds v among list[0 .. len) (stride `stride` elements).
__device__ __forceinline__ bool warp_contains(const uint32_t* __restrict__ list, uint64_t stride, uint32_t len,
                                              uint32_t v) {
  bool hit = false;
  for (uint32_t t = lane_id(); t < len; t += 32) hit |= (list[t * stride] == v);
  return __any_sync(0xFFFFFFFFu, hit);
}

__global__ void sample_fp_kernel(const uint32_t* __restrict__ pnn, uint64_t n, uint32_t k, uint32_t n_fp,
                                 uint64_t seed, uint32_t* __restrict__ out, uint32_t* __restrict__ err) {
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const uint32_t lane = lane_id();
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const uint32_t* reject = pnn + (i * k) * 2 + 1;  // column 1 of rows i*k .. (i+1)*k
    uint32_t* picks = out + (i * n_fp) * 2 + 1;      // column 1 of this point's output rows
    const bool self_in = warp_contains(reject, 2, k, static_cast<uint32_t>(i));
    uint64_t avail = n > k ? n - k : 0;
    const uint64_t self_cut = self_in ? 0 : 1;
    avail = avail > self_cut ? avail - self_cut : 0;
    const uint32_t want = static_cast<uint32_t>((n_fp < avail ? static_cast<uint64_t>(n_fp) : avail));
    PointStream s(seed, i);
    uint64_t budget = SAMPLE_ATTEMPT_CAP;
    uint32_t cnt = 0;
    while (cnt < want) {
      uint32_t j;
      if (!s.uniform(static_cast<uint32_t>(n), j, budget)) {
        if (lane == 0) atomicOr(err, DEV_ERR_SAMPLING);
        break;
      }
      if (j == i) continue;
      if (warp_contains(picks, 2, cnt, j) || warp_contains(reject, 2, k, j)) continue;
      if (lane == 0) {
        out[(i * n_fp + cnt) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_fp + cnt) * 2 + 1] = j;
      }
      __syncwarp();
      ++cnt;
    }
  }
}

// True when any lane holds v in one of its R registers of a lane-distributed list of `len` slots.
template <int R>
__device__ __forceinline__ bool reg_contains(const uint32_t (&reg)[R], uint32_t len, uint32_t v) {
  const uint32_t lane = lane_id();
  bool hit = false;
#pragma unroll
  for (int r = 0; r < R; ++r) hit |= (lane + 32u * r < len) && reg[r] == v;
  return __any_sync(0xFFFFFFFFu, hit);
}
template <int R>
__device__ __forceinline__ void reg_put(uint32_t (&reg)[R], uint32_t slot, uint32_t v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (lane + 32u * r == slot) reg[r] = v;
}

// sample_fp_kernel with the picks (n_fp <= 32 PR) and the k neighbours (k <= 32 RR) in registers.
template <int PR, int RR>
__global__ void sample_fp_reg_kernel(const uint32_t* __restrict__ pnn, uint64_t n, uint32_t k, uint32_t n_fp,
                                     uint64_t seed, uint32_t* __restrict__ out, uint32_t* __restrict__ err) {
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const uint32_t lane = lane_id();
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    uint32_t rej[RR], pk[PR];
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      const uint32_t t = lane + 32u * r;
      rej[r] = t < k ? pnn[((i * k) + t) * 2 + 1] : 0u;
    }
#pragma unroll
    for (int r = 0; r < PR; ++r) pk[r] = 0u;
    const bool self_in = reg_contains<RR>(rej, k, static_cast<uint32_t>(i));
    uint64_t avail = n > k ? n - k : 0;
    const uint64_t self_cut = self_in ? 0 : 1;
    avail = avail > self_cut ? avail - self_cut : 0;
    const uint32_t want = static_cast<uint32_t>((n_fp < avail ? static_cast<uint64_t>(n_fp) : avail));
    WarpStream s(seed, i);
    uint64_t budget = SAMPLE_ATTEMPT_CAP;
    uint32_t cnt = 0;
    while (cnt < want) {
      uint32_t j;
      if (!s.uniform(static_cast<uint32_t>(n), j, budget)) {
        if (lane == 0) atomicOr(err, DEV_ERR_SAMPLING);
        break;
      }
      if (j == i) continue;
      if (reg_contains<PR>(pk, cnt, j) || reg_contains<RR>(rej, k, j)) continue;
      reg_put<PR>(pk, cnt, j);
      if (lane == (cnt & 31u)) {
        out[(i * n_fp + cnt) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_fp + cnt) * 2 + 1] = j;
      }
      ++cnt;
    }
  }
}

// sample_fp_pair_deterministic 32 stream words at a time (k <= 64, n_fp <= 96, n < 2^31): lane L takes
// word pos + L of the point's stream (its own Philox block), applies the zone rule, and tests the value
// against i, the k neighbours and the earlier picks (both in shared memory); among the lanes that pass,
// only the first lane of each value counts (__match_any_sync), and the accepted lanes fill the slots
// in lane order. The words counted as used end at the lane that filled the last slot. This is the
// sequential rule of sample_fp_reg_kernel -- same picks, same order, same attempt budget -- with the
// per-draw votes replaced by independent work across the lanes.
constexpr int FPB_WARPS = 8, FPB_K = 64, FPB_P = 96;
__global__ void __launch_bounds__(FPB_WARPS * 32) sample_fp_batch_kernel(const uint32_t* __restrict__ pnn, uint64_t n,
                                                                         uint32_t k, uint32_t n_fp, uint64_t seed,
                                                                         uint32_t* __restrict__ out,
                                                                         uint32_t* __restrict__ err) {
  __shared__ uint32_t s_rej[FPB_WARPS][FPB_K];
  __shared__ uint32_t s_pk[FPB_WARPS][FPB_P];
  const int warp = threadIdx.x >> 5;
  const uint32_t lane = lane_id();
  uint32_t* rej = s_rej[warp];
  uint32_t* pk = s_pk[warp];
  const uint32_t range = static_cast<uint32_t>(n);
  const uint32_t zone = (range << __clz(range)) - 1u;
  const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * FPB_WARPS;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * FPB_WARPS + warp; i < n; i += warps) {
    __syncwarp();
    for (uint32_t t = lane; t < k; t += 32) rej[t] = pnn[((i * k) + t) * 2 + 1];
    __syncwarp();
    bool hit = false;
    for (uint32_t t = lane; t < k; t += 32) hit |= rej[t] == static_cast<uint32_t>(i);
    const bool self_in = __any_sync(0xFFFFFFFFu, hit);
    uint64_t avail = n > k ? n - k : 0;
    const uint64_t self_cut = self_in ? 0 : 1;
    avail = avail > self_cut ? avail - self_cut : 0;
    const uint32_t want = static_cast<uint32_t>((n_fp < avail ? static_cast<uint64_t>(n_fp) : avail));
    const uint32_t c1 = static_cast<uint32_t>(i), c2 = static_cast<uint32_t>(i >> 32);
    uint64_t pos = 0, budget = SAMPLE_ATTEMPT_CAP;
    uint32_t cnt = 0;
    while (cnt < want) {
      if (budget == 0) {
        if (lane == 0) atomicOr(err, DEV_ERR_SAMPLING);
        break;
      }
      const uint32_t avail_w = budget < 32 ? static_cast<uint32_t>(budget) : 32u;
      const uint64_t g = pos + lane;
      uint32_t w4[4];
      philox4x32_10(static_cast<uint32_t>(g >> 2), c1, c2, TAG_SAMPLE, k0, k1, w4);
      const uint32_t e = static_cast<uint32_t>(g & 3);
      const uint32_t w = e == 0 ? w4[0] : (e == 1 ? w4[1] : (e == 2 ? w4[2] : w4[3]));
      const uint32_t j = __umulhi(w, range);
      bool cand = lane < avail_w && w * range <= zone && j != static_cast<uint32_t>(i);
      if (__any_sync(0xFFFFFFFFu, cand)) {
        for (uint32_t t = 0; t < k; ++t) cand = cand && rej[t] != j;
        for (uint32_t t = 0; t < cnt; ++t) cand = cand && pk[t] != j;
      }
      const uint32_t key = cand ? j : (0x80000000u | lane);  // j < 2^31: sentinels never match a value
      const unsigned same = __match_any_sync(0xFFFFFFFFu, key);
      const bool acc = cand && lane == static_cast<uint32_t>(__ffs(same) - 1);
      const unsigned accm = __ballot_sync(0xFFFFFFFFu, acc);
      const uint32_t need = want - cnt, got = __popc(accm);
      const uint32_t rank = __popc(accm & ((1u << lane) - 1u));
      if (acc && rank < need) {
        pk[cnt + rank] = j;
        out[(i * n_fp + cnt + rank) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_fp + cnt + rank) * 2 + 1] = j;
      }
      uint32_t used = avail_w;
      if (got >= need) {
        const unsigned last = __ballot_sync(0xFFFFFFFFu, acc && rank == need - 1);
        used = static_cast<uint32_t>(__ffs(last));  // through the lane that filled the last slot
        cnt = want;
      } else {
        cnt += got;
      }
      pos += used;
      budget -= used;
      __syncwarp();
    }
  }
}

// The reference's f32 distance between rows a and b computed by an 8-lane group (l8 = lane % 8):
// lane l8 forms the lane accumulator l8 of distance.rs:60-66, the group sums them in order 0..7,
// adds the serial tail and takes the square root. Every lane of the group returns the result.
__device__ __forceinline__ float group8_ref_dist(const float* __restrict__ a, const float* __restrict__ b, int d,
                                                 int l8, unsigned group_base) {
  float acc = 0.0f;
  const int nc = d >> 3;
  for (int ch = 0; ch < nc; ++ch) {
    const float df = __fsub_rn(a[8 * ch + l8], b[8 * ch + l8]);
    acc = __fadd_rn(acc, __fmul_rn(df, df));
  }
  float t = 0.0f;
#pragma unroll
  for (int l = 0; l < 8; ++l) t = __fadd_rn(t, __shfl_sync(0xFFFFFFFFu, acc, group_base + l));
  for (int e = nc * 8; e < d; ++e) {
    const float df = __fsub_rn(a[e], b[e]);
    t = __fadd_rn(t, __fmul_rn(df, df));
  }
  return __fsqrt_rn(t);
}

// The mid-near pairs of point i by the reference's sequential rule (one warp; picks kept in `out`).
__device__ __noinline__ void mn_point_sequential(const float* __restrict__ x, uint64_t n, int d, uint32_t n_mn,
                                                 uint64_t seed, uint64_t i, uint32_t* __restrict__ out,
                                                 uint32_t* __restrict__ err) {
  const uint32_t lane = lane_id();
  const int l8 = lane & 7;
  const unsigned gbase = lane & ~7u;
  const int grp = lane >> 3;
  {
    uint32_t* picks = out + (i * n_mn) * 2 + 1;
    PointStream s(seed, i);
    uint64_t budget = SAMPLE_ATTEMPT_CAP;
    bool failed = false;
    for (uint32_t jslot = 0; jslot < n_mn && !failed; ++jslot) {
      const bool self_in = warp_contains(picks, 2, jslot, static_cast<uint32_t>(i));
      uint64_t avail = n > jslot ? n - jslot : 0;
      const uint64_t self_cut = self_in ? 0 : 1;
      avail = avail > self_cut ? avail - self_cut : 0;
      const uint32_t want = static_cast<uint32_t>((avail < 6 ? avail : 6ull));
      uint32_t cand[6] = {0, 0, 0, 0, 0, 0};
      uint32_t cnt = 0;
      while (cnt < want) {
        uint32_t j;
        if (!s.uniform(static_cast<uint32_t>(n), j, budget)) {
          failed = true;
          break;
        }
        if (j == i) continue;
        bool dup = false;
#pragma unroll
        for (int t = 0; t < 6; ++t) dup |= (t < static_cast<int>(cnt) && cand[t] == j);
        if (dup || warp_contains(picks, 2, jslot, j)) continue;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == static_cast<int>(cnt)) cand[t] = j;
        ++cnt;
      }
      if (failed) {
        if (lane == 0) atomicOr(err, DEV_ERR_SAMPLING);
        break;
      }
      // Distances of the drawn candidates: group g (lanes 8g..8g+7) handles slots g and g + 4.
      float dist[6];
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const int slot = pass * 4 + grp;
        float dv = 0.0f;
        uint32_t cidx = 0;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == slot) cidx = cand[t];
        const bool active = slot < static_cast<int>(cnt);
        // Groups with nothing to do still join the shuffles inside group8_ref_dist (on row i itself).
        const float r = group8_ref_dist(x + i * d, x + static_cast<uint64_t>(active ? cidx : i) * d, d, l8, gbase);
        dv = active ? r : 0.0f;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const float v = __shfl_sync(0xFFFFFFFFu, dv, g * 8);
          if (pass * 4 + g < 6) dist[pass * 4 + g] = v;
        }
      }
      // Slots >= cnt are the reference's (0.0, 0) fill. Pick the 2nd smallest (key, slot).
      uint64_t best0 = ~0ull, best1 = ~0ull;
      uint32_t id0 = 0, id1 = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const bool real = t < static_cast<int>(cnt);
        const float dv = real ? dist[t] : 0.0f;
        const uint32_t id = real ? cand[t] : 0u;
        const uint64_t key = (static_cast<uint64_t>(total_key(dv)) << 3) | static_cast<uint64_t>(t);
        if (key < best0) {
          best1 = best0;
          id1 = id0;
          best0 = key;
          id0 = id;
        } else if (key < best1) {
          best1 = key;
          id1 = id;
        }
      }
      if (lane == 0) {
        out[(i * n_mn + jslot) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_mn + jslot) * 2 + 1] = id1;
      }
      __syncwarp();
    }
  }
}

__global__ void sample_mn_kernel(const float* __restrict__ x, uint64_t n, int d, uint32_t n_mn, uint64_t seed,
                                 uint32_t* __restrict__ out, uint32_t* __restrict__ err) {
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps)
    mn_point_sequential(x, n, d, n_mn, seed, i, out, err);
}

// Speculative mid-near sampling (sampling.rs:118-142, 296-313), one warp per point, n_mn <= 32 and
// n >= n_mn + 7 (every slot then draws 6 candidates). The draws of every slot are made first, with the
// exclusion of the earlier slots' picks left out; then the 6 * n_mn candidate rows are gathered with many
// loads in flight (4 groups of 8 lanes, two rows each per pass; row i in NC registers per lane), each
// slot takes its 2nd-closest candidate, and the draws are checked: when no candidate of slot j is the
// pick of an earlier slot, the sequential rule would have accepted and rejected exactly the same stream
// words, so the picks are the rule's picks. Otherwise (rare: about 120 * n_mn / n per point) the point
// is redone by the sequential rule. Candidates and distances are staged in shared memory.
constexpr int MS_WARPS = 8, MS_MAXC = 32 * 6;
constexpr uint32_t MN_DRAW_BATCHES = 4;  // 512 words: 6 n_mn <= 192 draws need fewer unless n is tiny

// The rule's draws of all n_mn slots (6 candidates each) by the whole warp at once: lane L turns the four
// words of Philox block base + L into candidates (uniform by rejection, as PointStream::uniform, and the
// point itself skipped), and a prefix count over the lanes gives every accepted word its draw number, so
// draw p is the p-th accepted word -- the candidate the sequential loop assigns to slot p / 6, position
// p % 6, as long as no slot draws a point twice (the loop would skip the repeat and shift every later
// draw). Returns false when a slot holds a repeat or the batches ran out: the caller then runs the
// sequential rule for the point. cs receives 6 n_mn candidates in slot order.
__device__ __forceinline__ bool mn_draw_parallel(uint64_t seed, uint64_t i, uint32_t n, uint32_t n_mn,
                                                 uint32_t* __restrict__ cs) {
  const uint32_t lane = lane_id();
  const uint32_t total = n_mn * 6;
  const uint32_t zone = (n << __clz(n)) - 1u;
  const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
  const uint32_t c1 = static_cast<uint32_t>(i), c2 = static_cast<uint32_t>(i >> 32);
  uint32_t have = 0;
  for (uint32_t b = 0; b < MN_DRAW_BATCHES && have < total; ++b) {
    uint32_t w[4];
    philox4x32_10(b * 32u + lane, c1, c2, TAG_SAMPLE, k0, k1, w);
    uint32_t val[4], okm = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      val[t] = __umulhi(w[t], n);
      const bool ok = (w[t] * n <= zone) && (val[t] != static_cast<uint32_t>(i));
      okm |= (ok ? 1u : 0u) << t;
    }
    const uint32_t cnt = static_cast<uint32_t>(__popc(okm));
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<uint32_t>(o)) incl += v;
    }
    uint32_t p = have + incl - cnt;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if ((okm >> t) & 1u) {
        if (p < total) cs[p] = val[t];
        ++p;
      }
    }
    have += __shfl_sync(0xFFFFFFFFu, incl, 31);
  }
  __syncwarp();
  if (have < total) return false;
  bool dup = false;
  for (uint32_t sl = lane; sl < n_mn; sl += 32) {
    uint32_t c[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) c[t] = cs[sl * 6 + t];
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
      for (int b = a + 1; b < 6; ++b) dup |= c[a] == c[b];
  }
  return !__any_sync(0xFFFFFFFFu, dup);
}

template <int NC>
__global__ void __launch_bounds__(MS_WARPS * 32) sample_mn_spec_kernel(const float* __restrict__ x, uint64_t n, int d,
                                                                      uint32_t n_mn, uint64_t seed,
                                                                      uint32_t* __restrict__ out,
                                                                      uint32_t* __restrict__ err) {
  __shared__ uint32_t s_cand[MS_WARPS][MS_MAXC];
  __shared__ float s_dist[MS_WARPS][MS_MAXC];
  const int warp = threadIdx.x >> 5;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * MS_WARPS;
  const uint32_t lane = lane_id();
  const int l8 = lane & 7;
  const unsigned gbase = lane & ~7u;
  const int grp = lane >> 3;
  const int nc = d >> 3;
  const int total = static_cast<int>(n_mn) * 6;
  uint32_t* cs = s_cand[warp];
  float* ds = s_dist[warp];
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * MS_WARPS + warp; i < n; i += warps) {
    // 1. every slot's draws (self and repeats within the slot rejected, as in the rule), all words at once;
    //    a repeat within a slot (or words beyond the parallel batches) sends the point to the sequential rule
    if (!mn_draw_parallel(seed, i, static_cast<uint32_t>(n), n_mn, cs)) {
      mn_point_sequential(x, n, d, n_mn, seed, i, out, err);
      continue;
    }
    // 2. the reference's f32 distance of every candidate (distance.rs:50-75 order)
    const float* a = x + i * d;
    float ra[NC];
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) ra[ch] = ch < nc ? a[8 * ch + l8] : 0.0f;
    for (int c0 = 0; c0 < total; c0 += 8) {
      const int ca = c0 + grp, cb = c0 + 4 + grp;
      const uint32_t ja = ca < total ? cs[ca] : static_cast<uint32_t>(i);
      const uint32_t jb = cb < total ? cs[cb] : static_cast<uint32_t>(i);
      const float* pa = x + static_cast<uint64_t>(ja) * d;
      const float* pb = x + static_cast<uint64_t>(jb) * d;
      float va[NC], vb[NC];
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) {
        va[ch] = ch < nc ? pa[8 * ch + l8] : 0.0f;
        vb[ch] = ch < nc ? pb[8 * ch + l8] : 0.0f;
      }
      float acc_a = 0.0f, acc_b = 0.0f;
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) {
        if (ch < nc) {
          const float da = __fsub_rn(ra[ch], va[ch]), db = __fsub_rn(ra[ch], vb[ch]);
          acc_a = __fadd_rn(acc_a, __fmul_rn(da, da));
          acc_b = __fadd_rn(acc_b, __fmul_rn(db, db));
        }
      }
      float ta = 0.0f, tb = 0.0f;
#pragma unroll
      for (int l = 0; l < 8; ++l) {
        ta = __fadd_rn(ta, __shfl_sync(0xFFFFFFFFu, acc_a, gbase + l));
        tb = __fadd_rn(tb, __shfl_sync(0xFFFFFFFFu, acc_b, gbase + l));
      }
      for (int e = nc * 8; e < d; ++e) {
        const float da = __fsub_rn(a[e], pa[e]), db = __fsub_rn(a[e], pb[e]);
        ta = __fadd_rn(ta, __fmul_rn(da, da));
        tb = __fadd_rn(tb, __fmul_rn(db, db));
      }
      if (l8 == 0) {
        if (ca < total) ds[ca] = __fsqrt_rn(ta);
        if (cb < total) ds[cb] = __fsqrt_rn(tb);
      }
    }
    __syncwarp();
    // 3. lane j: slot j's 2nd smallest (distance key, draw order), then the check of its draws against the
    //    picks of the earlier slots
    uint32_t pick = 0;
    if (lane < n_mn) {
      uint64_t best0 = ~0ull, best1 = ~0ull;
      uint32_t id0 = 0, id1 = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const uint32_t id = cs[lane * 6 + t];
        const uint64_t key = (static_cast<uint64_t>(total_key(ds[lane * 6 + t])) << 3) | static_cast<uint64_t>(t);
        if (key < best0) {
          best1 = best0;
          id1 = id0;
          best0 = key;
          id0 = id;
        } else if (key < best1) {
          best1 = key;
          id1 = id;
        }
      }
      pick = id1;
    }
    bool clash = false;
    for (uint32_t q = 0; q + 1 < n_mn; ++q) {
      const uint32_t pq = __shfl_sync(0xFFFFFFFFu, pick, q);
      if (lane < n_mn && q < lane) {
#pragma unroll
        for (int t = 0; t < 6; ++t) clash |= cs[lane * 6 + t] == pq;
      }
    }
    __syncwarp();
    if (__any_sync(0xFFFFFFFFu, clash)) {
      mn_point_sequential(x, n, d, n_mn, seed, i, out, err);
      continue;
    }
    if (lane < n_mn) {
      out[(i * n_mn + lane) * 2 + 0] = static_cast<uint32_t>(i);
      out[(i * n_mn + lane) * 2 + 1] = pick;
    }
    __syncwarp();
  }
}

// The screened variant of sample_mn_spec_kernel (d a multiple of 16, at most 256): the candidates' rows
// are read from an fp16 copy h of x (half the bytes) with eps_j = |x_j - h_j| (rounded up) per row. By the
// triangle inequality the true distance lies within dist(x_i, h_j) -/+ eps_j, and the reference's f32
// distance within a further 2^-15 relative (its f32 sum over <= 256 terms, and this kernel's own). When
// those intervals settle both which two candidates are the closest and their order, the slot's pick is
// the reference's pick; otherwise the slot's six distances are computed exactly as distance.rs:50-75
// does. Exact ties always overlap, so they are always settled by the exact distances and the draw order.
constexpr float MN_REL = 3.0517578125e-05f;  // 2^-15
template <int E>  // elements per lane of the screening (d = 8 E)
__global__ void __launch_bounds__(MS_WARPS * 32, 3) sample_mn_screen_kernel(
    const float* __restrict__ x, const __half* __restrict__ h, const float* __restrict__ eps, uint64_t n, int d,
    uint32_t n_mn, uint64_t seed, uint32_t* __restrict__ out, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_cand[MS_WARPS][MS_MAXC];
  __shared__ float s_lo[MS_WARPS][MS_MAXC], s_hi[MS_WARPS][MS_MAXC];
  const int warp = threadIdx.x >> 5;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * MS_WARPS;
  const uint32_t lane = lane_id();
  const int l8 = lane & 7;
  const unsigned gbase = lane & ~7u;
  const int grp = lane >> 3;
  const int nc = d >> 3;
  const int total = static_cast<int>(n_mn) * 6;
  uint32_t* cs = s_cand[warp];
  float* lo_s = s_lo[warp];
  float* hi_s = s_hi[warp];
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * MS_WARPS + warp; i < n; i += warps) {
    // 1. every slot's draws (self and repeats within the slot rejected, as in the rule), all words at once;
    //    a repeat within a slot (or words beyond the parallel batches) sends the point to the sequential rule
    if (!mn_draw_parallel(seed, i, static_cast<uint32_t>(n), n_mn, cs)) {
      mn_point_sequential(x, n, d, n_mn, seed, i, out, err);
      continue;
    }
    // every candidate's fp16 row and bound towards L2 at once (the passes below then wait on L2, not on
    // one DRAM round trip per pass)
    {
      const int lines = (d * 2 + 127) / 128;
      for (int q = static_cast<int>(lane); q < total * lines; q += 32) {
        const int c = q / lines, ln = q - c * lines;
        const char* line = reinterpret_cast<const char*>(h + static_cast<uint64_t>(cs[c]) * d) + ln * 128;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
      }
      for (int c = static_cast<int>(lane); c < total; c += 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(eps + cs[c]));
    }
    // 2. screening distances on the fp16 rows: lane l8 of a group holds E consecutive elements (as E / 2
    //    pairs for the packed two-wide f32 arithmetic: even and odd elements are summed separately)
    const float* a = x + i * d;
    uint64_t xe[E / 2];
#pragma unroll
    for (int q = 0; q < E / 2; ++q) xe[q] = *reinterpret_cast<const uint64_t*>(a + l8 * E + 2 * q);
    for (int c0 = 0; c0 < total; c0 += 8) {
      const int ca = c0 + grp, cb = c0 + 4 + grp;
      const uint32_t ja = ca < total ? cs[ca] : static_cast<uint32_t>(i);
      const uint32_t jb = cb < total ? cs[cb] : static_cast<uint32_t>(i);
      const uint4* pa = reinterpret_cast<const uint4*>(h + static_cast<uint64_t>(ja) * d + l8 * E);
      const uint4* pb = reinterpret_cast<const uint4*>(h + static_cast<uint64_t>(jb) * d + l8 * E);
      uint4 va[E / 8], vb[E / 8];
#pragma unroll
      for (int q = 0; q < E / 8; ++q) {
        va[q] = pa[q];
        vb[q] = pb[q];
      }
      const float ea = eps[ja], eb = eps[jb];
      uint64_t pa2 = 0, pb2 = 0;  // (even, odd) partial sums
#pragma unroll
      for (int q = 0; q < E / 8; ++q) {
        const __half2* ha = reinterpret_cast<const __half2*>(&va[q]);
        const __half2* hb = reinterpret_cast<const __half2*>(&vb[q]);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const float2 fa = __half22float2(ha[w]), fb = __half22float2(hb[w]);
          const uint64_t da2 = f32x2_sub(xe[4 * q + w], f32x2_pack(fa)), db2 = f32x2_sub(xe[4 * q + w], f32x2_pack(fb));
          pa2 = f32x2_fma(da2, da2, pa2);
          pb2 = f32x2_fma(db2, db2, pb2);
        }
      }
      float sa = f32x2_lo(pa2) + f32x2_hi(pa2), sb = f32x2_lo(pb2) + f32x2_hi(pb2);
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xFFFFFFFFu, sa, o);
        sb += __shfl_xor_sync(0xFFFFFFFFu, sb, o);
      }
      if (l8 == 0) {
        const float da = sqrtf(sa), db = sqrtf(sb);
        // |ref - true| <= (d/8 + 12) 2^-24 true and |da - |x_i - h_j|| <= (d/2 + 8) 2^-24 da (two fused
        // multiply-add chains of d/16 terms per lane, 8 lanes, 3 shuffle sums, the final add, sqrt): 2^-15
        // covers both
        if (ca < total) {
          lo_s[ca] = da * (1.0f - MN_REL) - ea * (1.0f + MN_REL);
          hi_s[ca] = (da + ea) * (1.0f + MN_REL);
        }
        if (cb < total) {
          lo_s[cb] = db * (1.0f - MN_REL) - eb * (1.0f + MN_REL);
          hi_s[cb] = (db + eb) * (1.0f + MN_REL);
        }
      }
    }
    __syncwarp();
    // 3. lane j: slot j settled by the intervals? the two lowest upper bounds must lie below every other
    //    lower bound, and the lower of the two below the other's lower bound
    uint32_t pick = 0;
    bool exact = false;
    if (lane < n_mn) {
      float hi1 = 3.4e38f, hi2 = 3.4e38f;
      int t1 = 0, t2 = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const float hv = hi_s[lane * 6 + t];
        if (hv < hi1) {
          hi2 = hi1;
          t2 = t1;
          hi1 = hv;
          t1 = t;
        } else if (hv < hi2) {
          hi2 = hv;
          t2 = t;
        }
      }
      bool sure = hi1 < lo_s[lane * 6 + t2] && t1 != t2;
#pragma unroll
      for (int t = 0; t < 6; ++t)
        if (t != t1 && t != t2) sure = sure && hi2 < lo_s[lane * 6 + t];
      exact = !sure;
      pick = cs[lane * 6 + t2];
    }
    // 4. unsettled slots: the reference's exact distances of their six candidates (group g: slots t = g, g + 4)
    unsigned need = __ballot_sync(0xFFFFFFFFu, exact);
    while (need) {
      const int js = __ffs(need) - 1;
      need &= need - 1;
      float dist[6];
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const int t = pass * 4 + grp;
        const bool active = t < 6;
        const uint32_t cj = active ? cs[js * 6 + t] : static_cast<uint32_t>(i);
        const float r = group8_ref_dist(a, x + static_cast<uint64_t>(cj) * d, d, l8, gbase);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const float v = __shfl_sync(0xFFFFFFFFu, r, g * 8);
          if (pass * 4 + g < 6) dist[pass * 4 + g] = v;
        }
      }
      uint64_t best0 = ~0ull, best1 = ~0ull;
      uint32_t id1 = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const uint64_t key = (static_cast<uint64_t>(total_key(dist[t])) << 3) | static_cast<uint64_t>(t);
        if (key < best0) {
          best1 = best0;
          best0 = key;
        } else if (key < best1) {
          best1 = key;
        }
      }
      id1 = cs[js * 6 + static_cast<int>(best1 & 7u)];
      if (static_cast<int>(lane) == js) pick = id1;
    }
    (void)nc;
    // 5. the draws were made without the earlier picks: valid iff no candidate of slot j is a pick of a
    //    slot before j; otherwise the sequential rule redoes the point
    bool clash = false;
    for (uint32_t q = 0; q + 1 < n_mn; ++q) {
      const uint32_t pq = __shfl_sync(0xFFFFFFFFu, pick, q);
      if (lane < n_mn && q < lane) {
#pragma unroll
        for (int t = 0; t < 6; ++t) clash |= cs[lane * 6 + t] == pq;
      }
    }
    __syncwarp();
    if (__any_sync(0xFFFFFFFFu, clash)) {
      mn_point_sequential(x, n, d, n_mn, seed, i, out, err);
      continue;
    }
    if (lane < n_mn) {
      out[(i * n_mn + lane) * 2 + 0] = static_cast<uint32_t>(i);
      out[(i * n_mn + lane) * 2 + 1] = pick;
    }
    __syncwarp();
  }
}

// fp16 copy of x and each row's rounding-residual norm |x_j - h_j| (rounded up), one warp per row.
__global__ void half_rows_kernel(const float* __restrict__ x, uint64_t n, int d, __half* __restrict__ h,
                                 float* __restrict__ eps) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    float ss = 0.0f;
    for (int c = lane; c < d; c += 32) {
      const float v = x[r * d + c];
      const __half hv = __float2half_rn(v);
      h[r * d + c] = hv;
      const float res = v - __half2float(hv);  // exact (Sterbenz: hv is within a factor 2 of v, or both tiny)
      ss = fmaf(res, res, ss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xFFFFFFFFu, ss, o);
    // the f32 sum of d squares is within d 2^-24 relative, its square root within half that: 2^-15 covers both
    if (lane == 0) eps[r] = sqrtf(ss) * (1.0f + MN_REL) + 1e-30f;
  }
}

// sample_mn_kernel with the picks (n_mn <= 32) in one register per lane and row i of x (d <= 8 NC)
// in NC registers of each 8-lane group.
template <int NC>
__global__ void __launch_bounds__(256, NC <= 16 ? 4 : 3) sample_mn_reg_kernel(const float* __restrict__ x, uint64_t n, int d, uint32_t n_mn, uint64_t seed,
                                     uint32_t* __restrict__ out, uint32_t* __restrict__ err) {
  const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
  const uint32_t lane = lane_id();
  const int l8 = lane & 7;
  const unsigned gbase = lane & ~7u;
  const int grp = lane >> 3;
  const int nc = d >> 3;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const float* a = x + i * d;
    float ra[NC];
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) ra[ch] = ch < nc ? a[8 * ch + l8] : 0.0f;
    uint32_t pk[1] = {0u};
    WarpStream s(seed, i);
    uint64_t budget = SAMPLE_ATTEMPT_CAP;
    bool failed = false;
    for (uint32_t jslot = 0; jslot < n_mn && !failed; ++jslot) {
      const bool self_in = reg_contains<1>(pk, jslot, static_cast<uint32_t>(i));
      uint64_t avail = n > jslot ? n - jslot : 0;
      const uint64_t self_cut = self_in ? 0 : 1;
      avail = avail > self_cut ? avail - self_cut : 0;
      const uint32_t want = static_cast<uint32_t>((avail < 6 ? avail : 6ull));
      uint32_t cand[6] = {0, 0, 0, 0, 0, 0};
      uint32_t cnt = 0;
      while (cnt < want) {
        uint32_t j;
        if (!s.uniform(static_cast<uint32_t>(n), j, budget)) {
          failed = true;
          break;
        }
        if (j == i) continue;
        bool dup = false;
#pragma unroll
        for (int t = 0; t < 6; ++t) dup |= (t < static_cast<int>(cnt) && cand[t] == j);
        if (dup || reg_contains<1>(pk, jslot, j)) continue;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == static_cast<int>(cnt)) cand[t] = j;
        ++cnt;
      }
      if (failed) {
        if (lane == 0) atomicOr(err, DEV_ERR_SAMPLING);
        break;
      }
      // The candidates' rows are random HBM reads: start all of them towards L2 now (one 128-byte line
      // per lane and step), so the second pass below finds its rows there.
      {
        const int lines = (d * 4 + 127) / 128;
        for (int q = static_cast<int>(lane); q < static_cast<int>(cnt) * lines; q += 32) {
          const int slot = q / lines, ln = q - slot * lines;
          uint32_t cj = 0;
#pragma unroll
          for (int t = 0; t < 6; ++t)
            if (t == slot) cj = cand[t];
          const char* line = reinterpret_cast<const char*>(x + static_cast<uint64_t>(cj) * d) + ln * 128;
          asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
        }
      }
      // Distances of the drawn candidates in the reference's order (group8_ref_dist with row i in
      // registers): group g (lanes 8g..8g+7) handles slots g and g + 4.
      float dist[6];
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const int slot = pass * 4 + grp;
        uint32_t cidx = 0;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == slot) cidx = cand[t];
        const bool active = slot < static_cast<int>(cnt);
        const float* b = x + static_cast<uint64_t>(active ? cidx : i) * d;
        float acc = 0.0f;
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
          if (ch < nc) {
            const float df = __fsub_rn(ra[ch], b[8 * ch + l8]);
            acc = __fadd_rn(acc, __fmul_rn(df, df));
          }
        }
        float tsum = 0.0f;
#pragma unroll
        for (int l = 0; l < 8; ++l) tsum = __fadd_rn(tsum, __shfl_sync(0xFFFFFFFFu, acc, gbase + l));
        for (int e = nc * 8; e < d; ++e) {
          const float df = __fsub_rn(a[e], b[e]);
          tsum = __fadd_rn(tsum, __fmul_rn(df, df));
        }
        const float dv = active ? __fsqrt_rn(tsum) : 0.0f;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const float vv = __shfl_sync(0xFFFFFFFFu, dv, g * 8);
          if (pass * 4 + g < 6) dist[pass * 4 + g] = vv;
        }
      }
      // Slots >= cnt are the reference's (0.0, 0) fill. Pick the 2nd smallest (key, slot).
      uint64_t best0 = ~0ull, best1 = ~0ull;
      uint32_t id0 = 0, id1 = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const bool real = t < static_cast<int>(cnt);
        const float dv = real ? dist[t] : 0.0f;
        const uint32_t id = real ? cand[t] : 0u;
        const uint64_t key = (static_cast<uint64_t>(total_key(dv)) << 3) | static_cast<uint64_t>(t);
        if (key < best0) {
          best1 = best0;
          id1 = id0;
          best0 = key;
          id0 = id;
        } else if (key < best1) {
          best1 = key;
          id1 = id;
        }
      }
      reg_put<1>(pk, jslot, id1);
      if (lane == 0) {
        out[(i * n_mn + jslot) * 2 + 0] = static_cast<uint32_t>(i);
        out[(i * n_mn + jslot) * 2 + 1] = id1;
      }
    }
  }
}

}  // namespace

void sigma_device(Ctx& c, const float* d_kd, uint64_t n, uint64_t kp, float* d_sig) {
  sigma_kernel<<<ceil_div(n, 256), 256, 0, c.stream>>>(d_kd, n, static_cast<int>(kp), d_sig);
  PM_LAUNCHED();
}

void reselect_device(Ctx& c, const uint32_t* d_nbr, const float* d_kd, const float* d_sig, uint64_t n, uint64_t kp,
                     uint64_t k, uint32_t* d_pnn) {
  if (n == 0 || k == 0) return;
  PM_REQUIRE(kp <= 4096 && k <= kp, PACMAP_ERR_UNSUPPORTED, "neighbour reselection supports k' <= 4096");
  const int P = next_pow2(static_cast<int>(kp));
  const size_t smem = static_cast<size_t>(RS_WARPS) * P * sizeof(uint64_t);
  PM_CUDA(cudaFuncSetAttribute(reselect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n, RS_WARPS), c.sm_count * 16ull));
  reselect_kernel<<<grid, RS_WARPS * 32, smem, c.stream>>>(d_nbr, d_kd, d_sig, n, static_cast<int>(kp),
                                                           static_cast<int>(k), P, d_pnn);
  PM_LAUNCHED();
}

void sample_fp_device(Ctx& c, const uint32_t* d_pnn, uint64_t n, uint64_t k, uint64_t n_fp, uint64_t seed,
                      uint32_t* d_pfp) {
  if (n == 0 || n_fp == 0) return;
  PM_REQUIRE(n < (1ull << 32), PACMAP_ERR_UNSUPPORTED, "pair indices are u32: n must be < 2^32");
  PM_CUDA(cudaMemsetAsync(d_pfp, 0, n * n_fp * 2 * sizeof(uint32_t), c.stream));
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n, 8), c.sm_count * 32ull));
  const uint32_t k32 = static_cast<uint32_t>(k), f32n = static_cast<uint32_t>(n_fp);
  if (n_fp <= static_cast<uint64_t>(FPB_P) && k <= static_cast<uint64_t>(FPB_K) && n < (1ull << 31))
    sample_fp_batch_kernel<<<grid, FPB_WARPS * 32, 0, c.stream>>>(d_pnn, n, k32, f32n, seed, d_pfp, c.d_err);
  else if (n_fp <= 96 && k <= 64)
    sample_fp_reg_kernel<3, 2><<<grid, 256, 0, c.stream>>>(d_pnn, n, k32, f32n, seed, d_pfp, c.d_err);
  else if (n_fp <= 256 && k <= 128)
    sample_fp_reg_kernel<8, 4><<<grid, 256, 0, c.stream>>>(d_pnn, n, k32, f32n, seed, d_pfp, c.d_err);
  else
    sample_fp_kernel<<<grid, 256, 0, c.stream>>>(d_pnn, n, k32, f32n, seed, d_pfp, c.d_err);
  PM_LAUNCHED();
}

void sample_mn_device(Ctx& c, const float* d_xp, uint64_t n, uint64_t d, uint64_t n_mn, uint64_t seed,
                      uint32_t* d_pmn) {
  if (n == 0 || n_mn == 0) return;
  PM_REQUIRE(n < (1ull << 32), PACMAP_ERR_UNSUPPORTED, "pair indices are u32: n must be < 2^32");
  PM_CUDA(cudaMemsetAsync(d_pmn, 0, n * n_mn * 2 * sizeof(uint32_t), c.stream));
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div(n, 8), c.sm_count * 32ull));
  const int di = static_cast<int>(d);
  const uint32_t m32 = static_cast<uint32_t>(n_mn);
  const bool spec = n_mn <= 32 && n >= n_mn + 7;
  if (spec && (d == 128 || d == 256)) {
    // screened on an fp16 copy (half the gathered bytes); the unsettled slots use the exact rows
    DevBuf<__half> h(c, n * d);
    DevBuf<float> eps(c, n);
    half_rows_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(n, 8), c.sm_count * 32ull)), 256, 0,
                       c.stream>>>(d_xp, n, di, h.get(), eps.get());
    PM_LAUNCHED();
    if (d == 128)
      sample_mn_screen_kernel<16><<<grid, MS_WARPS * 32, 0, c.stream>>>(d_xp, h.get(), eps.get(), n, di, m32, seed,
                                                                         d_pmn, c.d_err);
    else
      sample_mn_screen_kernel<32><<<grid, MS_WARPS * 32, 0, c.stream>>>(d_xp, h.get(), eps.get(), n, di, m32, seed,
                                                                         d_pmn, c.d_err);
    PM_LAUNCHED();
    return;
  }
  if (spec && d <= 128)
    sample_mn_spec_kernel<16><<<grid, MS_WARPS * 32, 0, c.stream>>>(d_xp, n, di, m32, seed, d_pmn, c.d_err);
  else if (spec && d <= 256)
    sample_mn_spec_kernel<32><<<grid, MS_WARPS * 32, 0, c.stream>>>(d_xp, n, di, m32, seed, d_pmn, c.d_err);
  else if (n_mn <= 32 && d <= 128)
    sample_mn_reg_kernel<16><<<grid, 256, 0, c.stream>>>(d_xp, n, di, m32, seed, d_pmn, c.d_err);
  else if (n_mn <= 32 && d <= 256)
    sample_mn_reg_kernel<32><<<grid, 256, 0, c.stream>>>(d_xp, n, di, m32, seed, d_pmn, c.d_err);
  else
    sample_mn_kernel<<<grid, 256, 0, c.stream>>>(d_xp, n, di, m32, seed, d_pmn, c.d_err);
  PM_LAUNCHED();
}

}  // namespace pacmap
