// The learned initialiser (no reference analogue; it lets a shortened schedule replace the plain one): an MLP
// d -> 512 -> 512 -> dim (ReLU) with BF16 weights and activations and FP32 accumulation, trained with
// AdamW on (preprocessed x, PaCMAP embedding) pairs and applied to new data as Initialization::Value
// (src/lib.rs:753-766 rescales it to std 1e-4, so only its geometry matters).
//
// Every GEMM of the forward and backward pass is one hand-written tcgen05 kernel, C = A . B^T with
// both operands K-major BF16 (TMA, 128-byte swizzle, 4-stage pipeline, FP32 accumulator in TMEM) and a
// fused epilogue: bias + ReLU -> BF16, ReLU backprop through the stored activation -> BF16, or FP32.
// Operands needed in the other orientation (X^T, H^T, dZ^T, W^T) come from a BF16 transpose kernel.
// FP32 master weights, AdamW (decoupled weight decay), BF16 copies refreshed after each step.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "engine.cuh"
#include "mlp.cuh"
#include "tcgen05.cuh"

namespace pacmap {
namespace {

constexpr int MLP_H = 512;
constexpr int GEMM_THREADS = 192;  // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2..5 epilogue
constexpr int GEMM_STAGES = 2;  // 66 KB at BN = 128: three blocks per SM overlap each other's epilogues
constexpr int A_STAGE = 128 * 128;  // 128 rows x 64 bf16

enum Epi : int { EPI_F32 = 0, EPI_BIAS_RELU = 1, EPI_DRELU = 2 };

struct GemmOut {
  float* out_f32;
  __nv_bfloat16* out_bf16;
  const float* bias;
  const __nv_bfloat16* aux;  // the forward activation H (ReLU'(Z) = H > 0)
  int ld_out, ld_aux, m_valid, n_valid;
};

struct alignas(8) GemmShared {
  uint64_t full[GEMM_STAGES];
  uint64_t empty[GEMM_STAGES];
  uint64_t done;
  uint32_t tmem_base;
  int abort_flag;
};

template <int BN>
__host__ __device__ constexpr int tmem_cols() {
  return BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
}

template <int BN, int EPI>
__global__ void __launch_bounds__(GEMM_THREADS, 1) gemm_tn_kernel(const __grid_constant__ CUtensorMap amap,
                                                                  const __grid_constant__ CUtensorMap bmap, int K,
                                                                  GemmOut o, uint32_t* __restrict__ err) {
  constexpr int B_STAGE = BN * 128;
  extern __shared__ __align__(1024) unsigned char gemm_raw[];
  // aligned by offsetting the shared array itself, so every access keeps the shared address space
  unsigned char* base = gemm_raw + ((1024u - (smem_u32(gemm_raw) & 1023u)) & 1023u);
  unsigned char* a_s = base;
  unsigned char* b_s = base + GEMM_STAGES * A_STAGE;
  GemmShared* sh = reinterpret_cast<GemmShared*>(b_s + GEMM_STAGES * B_STAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
  const int nk = K / 64;
  if (threadIdx.x == 0) {
    for (int s = 0; s < GEMM_STAGES; ++s) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 1);
    }
    mbar_init(&sh->done, 1);
    sh->abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"(tmem_cols<BN>()));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;
  volatile int* abort_flag = &sh->abort_flag;
  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % GEMM_STAGES;
        if (kb >= GEMM_STAGES && !mbar_wait(&sh->empty[s], ((kb / GEMM_STAGES) + 1) & 1, abort_flag)) break;
        mbar_expect_tx(&sh->full[s], A_STAGE + B_STAGE);
        tma_load_2d(a_s + s * A_STAGE, &amap, &sh->full[s], kb * 64, m0);
        tma_load_2d(b_s + s * B_STAGE, &bmap, &sh->full[s], kb * 64, n0);
        issued = kb + 1;
      }
      if (issued < nk) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      for (int kb = (issued > GEMM_STAGES ? issued - GEMM_STAGES : 0); kb < issued; ++kb) {
        const uint64_t t0 = globaltimer();
        while (!mbar_try_wait(&sh->full[kb % GEMM_STAGES], (kb / GEMM_STAGES) & 1) && globaltimer() - t0 < WAIT_LIMIT_NS) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_f16_mn(true, BN);
      bool ok = true;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % GEMM_STAGES;
        if (!mbar_wait(&sh->full[s], (kb / GEMM_STAGES) & 1, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t ad = sdesc_sw128(smem_u32(a_s + s * A_STAGE));
        const uint64_t bd = sdesc_sw128(smem_u32(b_s + s * B_STAGE));
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) umma_f16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) ? 1u : 0u);
        umma_commit(&sh->empty[s]);
      }
      if (!ok) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        sh->abort_flag = 1;
      }
      umma_commit(&sh->done);
      // Every issued MMA has completed before the tensor memory is released (bounded, whatever the abort
      // flag: the epilogue's own wait gives up at once on abort).
      const uint64_t t0 = globaltimer();
      while (!mbar_try_wait(&sh->done, 0) && globaltimer() - t0 < WAIT_LIMIT_NS) {
      }
    }
  } else {
    const int quad = warp & 3;
    const int row = m0 + quad * 32 + lane;
    if (mbar_wait(&sh->done, 0, abort_flag) && !*abort_flag) {
      tc_fence_after();
      const uint32_t taddr = tmem + (static_cast<uint32_t>(quad * 32) << 16);
      constexpr int CH = BN < 32 ? BN : 32;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += CH) {
        float v[32];
        if constexpr (CH == 32) {
          tmem_ld32(taddr + c0, v);
        } else {
          float w[16];
          tmem_ld16(taddr + c0, w);
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] = w[i];
        }
        if (row < o.m_valid) {
          if (EPI != EPI_F32 && CH == 32 && n0 + c0 + 32 <= o.n_valid && (o.ld_out % 8) == 0 &&
              (EPI != EPI_DRELU || (o.ld_aux % 8) == 0)) {
            // 32 bf16 of this row: four 16-byte stores (and four 16-byte loads of the activation)
            const size_t off = static_cast<size_t>(row) * o.ld_out + n0 + c0;
            uint4* dst = reinterpret_cast<uint4*>(o.out_bf16 + off);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              uint32_t w[4];
              uint4 hv = make_uint4(0u, 0u, 0u, 0u);
              if (EPI == EPI_DRELU)
                hv = *reinterpret_cast<const uint4*>(o.aux + static_cast<size_t>(row) * o.ld_aux + n0 + c0 + 8 * q);
              const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                float lo = v[8 * q + 2 * e], hi = v[8 * q + 2 * e + 1];
                if (EPI == EPI_BIAS_RELU) {
                  lo += o.bias[n0 + c0 + 8 * q + 2 * e];
                  hi += o.bias[n0 + c0 + 8 * q + 2 * e + 1];
                  lo = lo > 0.0f ? lo : 0.0f;
                  hi = hi > 0.0f ? hi : 0.0f;
                } else {
                  const float hl = __uint_as_float(hw[e] << 16), hh = __uint_as_float(hw[e] & 0xFFFF0000u);
                  lo = hl > 0.0f ? lo : 0.0f;
                  hi = hh > 0.0f ? hi : 0.0f;
                }
                w[e] = static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(lo))) |
                       (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(hi))) << 16);
              }
              dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
            }
          } else {
#pragma unroll
            for (int i = 0; i < CH; ++i) {
              const int col = n0 + c0 + i;
              if (col >= o.n_valid) continue;
              float a = v[i];
              const size_t off = static_cast<size_t>(row) * o.ld_out + col;
              if (EPI == EPI_F32) {
                if (o.bias) a += o.bias[col];
                o.out_f32[off] = a;
              } else if (EPI == EPI_BIAS_RELU) {
                a += o.bias[col];
                o.out_bf16[off] = __float2bfloat16_rn(a > 0.0f ? a : 0.0f);
              } else {
                const float h = __bfloat162float(o.aux[static_cast<size_t>(row) * o.ld_aux + col]);
                o.out_bf16[off] = __float2bfloat16_rn(h > 0.0f ? a : 0.0f);
              }
            }
          }
        }
      }
    } else {
      atomicOr(err, DEV_ERR_TIMEOUT);
      sh->abort_flag = 1;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols<BN>()));
}

// f32 rows (optionally gathered through `rows`) -> bf16 [rows_pad][cols_pad], zero padded.
__global__ void cast_pad_kernel(const float* __restrict__ src, const uint32_t* __restrict__ rows, uint64_t n_rows,
                                int cols, int ld_src, uint64_t rows_pad, int cols_pad, __nv_bfloat16* __restrict__ dst) {
  const uint64_t total = rows_pad * cols_pad;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const uint64_t r = t / cols_pad;
    const int c = static_cast<int>(t % cols_pad);
    float v = 0.0f;
    if (r < n_rows && c < cols) v = src[(rows ? static_cast<uint64_t>(rows[r]) : r) * ld_src + c];
    dst[t] = __float2bfloat16_rn(v);
  }
}

// bf16 [R][C] -> bf16 [C][R] (32 x 32 tiles through shared memory).
__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ src, int R, int C,
                                      __nv_bfloat16* __restrict__ dst) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < R && c < C) ? src[static_cast<size_t>(r) * C + c] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < C && r < R) dst[static_cast<size_t>(c) * R + r] = tile[threadIdx.x][i];
  }
}

// MSE: out [B][ld_out] (first `dim` columns), target [B][dim] -> dZ = 2 (out - t) / (B dim) as bf16
// [B][ld_dz] (zero padded) and per-block partial sums of squared errors.
__global__ void mse_grad_kernel(const float* __restrict__ out, int ld_out, const float* __restrict__ target, int B,
                                int dim, int ld_dz, __nv_bfloat16* __restrict__ dz, double* __restrict__ partial) {
  __shared__ double red[256];
  double s = 0.0;
  const float scale = 2.0f / static_cast<float>(B * dim);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < B * ld_dz; t += gridDim.x * blockDim.x) {
    const int r = t / ld_dz, c = t % ld_dz;
    float g = 0.0f;
    if (c < dim) {
      const float e = out[static_cast<size_t>(r) * ld_out + c] - target[static_cast<size_t>(r) * dim + c];
      s += static_cast<double>(e) * e;
      g = scale * e;
    }
    dz[t] = __float2bfloat16_rn(g);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Column sums of the first C columns of a bf16 [R][ld] matrix (bias gradients), one thread per
// column in row order.
__global__ void colsum_bf16_kernel(const __nv_bfloat16* __restrict__ src, int R, int C, int ld,
                                   float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.0f;
  for (int r = 0; r < R; ++r) s += __bfloat162float(src[static_cast<size_t>(r) * ld + c]);
  out[c] = s;
}

// dst[r][c] = src[rows[r]][c] (f32, dim columns).
__global__ void gather_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ rows, uint64_t n_rows,
                                   int dim, float* __restrict__ dst) {
  const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n_rows * dim) return;
  const uint64_t r = t / dim;
  dst[t] = src[static_cast<uint64_t>(rows[r]) * dim + (t % dim)];
}

// AdamW (decoupled weight decay) on an f32 master tensor; also writes its bf16 copy.
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                             float* __restrict__ v, uint64_t count, float lr, float wd, float b1c, float b2c,
                             __nv_bfloat16* __restrict__ pb) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride) {
    const float gg = g[t];
    float mm = 0.9f * m[t] + 0.1f * gg;
    float vv = 0.999f * v[t] + 0.001f * gg * gg;
    m[t] = mm;
    v[t] = vv;
    float w = p[t] * (1.0f - lr * wd);
    w -= lr * (mm / b1c) / (sqrtf(vv / b2c) + 1e-8f);
    p[t] = w;
    if (pb) pb[t] = __float2bfloat16_rn(w);
  }
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ src, uint64_t count, __nv_bfloat16* __restrict__ dst) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride)
    dst[t] = __float2bfloat16_rn(src[t]);
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
inline int pad_to(int v, int m) { return (v + m - 1) / m * m; }

template <int BN, int EPI>
void gemm(Ctx& c, const __nv_bfloat16* A, int M_rows_alloc, const __nv_bfloat16* Bm, int N_rows_alloc, int K,
          const GemmOut& o) {
  const CUtensorMap am = make_tmap_2d_16b(A, M_rows_alloc, K, 128, true);
  const CUtensorMap bm = make_tmap_2d_16b(Bm, N_rows_alloc, K, BN, true);
  const size_t smem = 1024 + GEMM_STAGES * (A_STAGE + BN * 128) + sizeof(GemmShared);
  PM_CUDA(cudaFuncSetAttribute(gemm_tn_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)));
  const dim3 grid(static_cast<unsigned>(M_rows_alloc / 128), static_cast<unsigned>((N_rows_alloc + BN - 1) / BN));
  gemm_tn_kernel<BN, EPI><<<grid, GEMM_THREADS, smem, c.stream>>>(am, bm, K, o, c.d_err);
  PM_LAUNCHED();
}

void transpose(Ctx& c, const __nv_bfloat16* src, int R, int C, __nv_bfloat16* dst) {
  transpose_bf16_kernel<<<dim3(ceil_div(C, 32), ceil_div(R, 32)), dim3(32, 8), 0, c.stream>>>(src, R, C, dst);
  PM_LAUNCHED();
}

void cast_pad(Ctx& c, const float* src, const uint32_t* rows, uint64_t n_rows, int cols, int ld_src,
              uint64_t rows_pad, int cols_pad, __nv_bfloat16* dst) {
  const uint64_t total = rows_pad * cols_pad;
  cast_pad_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(total, 256), c.sm_count * 16ull)), 256, 0,
                    c.stream>>>(src, rows, n_rows, cols, ld_src, rows_pad, cols_pad, dst);
  PM_LAUNCHED();
}

}  // namespace

// Network state on the device: f32 masters in GEMM-friendly layouts, their bf16 copies and moments.
struct MlpNet {
  int d = 0, dp = 0, dim = 0, dp16 = 16, dp64 = 64;
  DevBuf<float> W1, b1, W2, b2, W3T, b3;            // W1 [512][dp], W2 [512][512], W3T [512][dp16], b3 [dp16]
  DevBuf<__nv_bfloat16> W1b, W2b, W3b, W2Tb, W3Tb;   // W3b [dp16][512], W2Tb [512][512], W3Tb [512][dp64]
  void alloc(Ctx& c, int d_, int dim_) {
    d = d_;
    dim = dim_;
    dp = pad_to(d, 64);
    dp16 = pad_to(dim, 16);
    dp64 = pad_to(dim, 64);
    W1.alloc(c, static_cast<size_t>(MLP_H) * dp);
    b1.alloc(c, MLP_H);
    W2.alloc(c, static_cast<size_t>(MLP_H) * MLP_H);
    b2.alloc(c, MLP_H);
    W3T.alloc(c, static_cast<size_t>(MLP_H) * dp16);
    b3.alloc(c, dp16);
    W1b.alloc(c, W1.count);
    W2b.alloc(c, W2.count);
    W3b.alloc(c, static_cast<size_t>(dp16) * MLP_H);
    W2Tb.alloc(c, W2.count);
    W3Tb.alloc(c, static_cast<size_t>(MLP_H) * dp64);
  }
  // flat host layout [W1 (512 x d), b1, W2 (512 x 512), b2, W3 (dim x 512), b3] <-> device layouts
  void upload(Ctx& c, const float* flat) {
    std::vector<float> w1(W1.count, 0.0f), w3t(W3T.count, 0.0f), bb3(dp16, 0.0f);
    const float* p = flat;
    for (int j = 0; j < MLP_H; ++j)
      for (int i = 0; i < d; ++i) w1[static_cast<size_t>(j) * dp + i] = p[static_cast<size_t>(j) * d + i];
    p += static_cast<size_t>(MLP_H) * d;
    PM_CUDA(cudaMemcpyAsync(W1.get(), w1.data(), W1.bytes(), cudaMemcpyHostToDevice, c.stream));
    PM_CUDA(cudaMemcpyAsync(b1.get(), p, MLP_H * 4, cudaMemcpyHostToDevice, c.stream));
    p += MLP_H;
    PM_CUDA(cudaMemcpyAsync(W2.get(), p, W2.bytes(), cudaMemcpyHostToDevice, c.stream));
    p += static_cast<size_t>(MLP_H) * MLP_H;
    PM_CUDA(cudaMemcpyAsync(b2.get(), p, MLP_H * 4, cudaMemcpyHostToDevice, c.stream));
    p += MLP_H;
    for (int k = 0; k < dim; ++k)
      for (int i = 0; i < MLP_H; ++i) w3t[static_cast<size_t>(i) * dp16 + k] = p[static_cast<size_t>(k) * MLP_H + i];
    p += static_cast<size_t>(dim) * MLP_H;
    for (int k = 0; k < dim; ++k) bb3[k] = p[k];
    PM_CUDA(cudaMemcpyAsync(W3T.get(), w3t.data(), W3T.bytes(), cudaMemcpyHostToDevice, c.stream));
    PM_CUDA(cudaMemcpyAsync(b3.get(), bb3.data(), b3.bytes(), cudaMemcpyHostToDevice, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    refresh(c);
  }
  void download(Ctx& c, float* flat) {
    std::vector<float> w1(W1.count), w3t(W3T.count), bb3(dp16);
    PM_CUDA(cudaMemcpyAsync(w1.data(), W1.get(), W1.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(w3t.data(), W3T.get(), W3T.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(bb3.data(), b3.get(), b3.bytes(), cudaMemcpyDeviceToHost, c.stream));
    float* p = flat;
    float* pb1 = p + static_cast<size_t>(MLP_H) * d;
    float* pW2 = pb1 + MLP_H;
    float* pb2 = pW2 + static_cast<size_t>(MLP_H) * MLP_H;
    float* pW3 = pb2 + MLP_H;
    float* pb3 = pW3 + static_cast<size_t>(dim) * MLP_H;
    PM_CUDA(cudaMemcpyAsync(pb1, b1.get(), MLP_H * 4, cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(pW2, W2.get(), W2.bytes(), cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaMemcpyAsync(pb2, b2.get(), MLP_H * 4, cudaMemcpyDeviceToHost, c.stream));
    PM_CUDA(cudaStreamSynchronize(c.stream));
    for (int j = 0; j < MLP_H; ++j)
      for (int i = 0; i < d; ++i) p[static_cast<size_t>(j) * d + i] = w1[static_cast<size_t>(j) * dp + i];
    for (int k = 0; k < dim; ++k)
      for (int i = 0; i < MLP_H; ++i) pW3[static_cast<size_t>(k) * MLP_H + i] = w3t[static_cast<size_t>(i) * dp16 + k];
    for (int k = 0; k < dim; ++k) pb3[k] = bb3[k];
  }
  // bf16 copies in the operand layouts: W1b = W1, W2b = W2, W2Tb = W2^T, W3b = W3 [dp16][512] (=W3T^T),
  // W3Tb = W3T padded to dp64 columns.
  void refresh(Ctx& c) {
    f32_to_bf16_kernel<<<256, 256, 0, c.stream>>>(W1.get(), W1.count, W1b.get());
    PM_LAUNCHED();
    f32_to_bf16_kernel<<<256, 256, 0, c.stream>>>(W2.get(), W2.count, W2b.get());
    PM_LAUNCHED();
    transpose(c, W2b.get(), MLP_H, MLP_H, W2Tb.get());
    DevBuf<__nv_bfloat16> w3tb(c, W3T.count);
    f32_to_bf16_kernel<<<64, 256, 0, c.stream>>>(W3T.get(), W3T.count, w3tb.get());
    PM_LAUNCHED();
    transpose(c, w3tb.get(), MLP_H, dp16, W3b.get());
    cast_pad(c, W3T.get(), nullptr, MLP_H, dp16, dp16, MLP_H, dp64, W3Tb.get());
  }
};

namespace {

// Forward through the network: X bf16 [rows][dp] (rows a multiple of 128) -> H1, H2 bf16 [rows][512],
// out f32 [rows][dp16].
void mlp_forward(Ctx& c, MlpNet& net, const __nv_bfloat16* X, int rows, __nv_bfloat16* H1, __nv_bfloat16* H2,
                 float* out, int m_valid) {
  GemmOut o{};
  o.bias = net.b1.get();
  o.out_bf16 = H1;
  o.ld_out = MLP_H;
  o.m_valid = m_valid;
  o.n_valid = MLP_H;
  gemm<128, EPI_BIAS_RELU>(c, X, rows, net.W1b.get(), MLP_H, net.dp, o);
  o.bias = net.b2.get();
  o.out_bf16 = H2;
  gemm<128, EPI_BIAS_RELU>(c, H1, rows, net.W2b.get(), MLP_H, MLP_H, o);
  GemmOut f{};
  f.bias = net.b3.get();
  f.out_f32 = out;
  f.ld_out = net.dp16;
  f.m_valid = m_valid;
  f.n_valid = net.dp16;
  gemm<16, EPI_F32>(c, H2, rows, net.W3b.get(), net.dp16, MLP_H, f);
}

// Scratch for one batch of B rows.
struct MlpBatch {
  int B = 0;
  DevBuf<__nv_bfloat16> X, XT, H1, H1T, H2, H2T, dZ3, dZ3T, dZ2, dZ2T, dZ1, dZ1T;
  DevBuf<float> out, tgt, gW1, gb1, gW2, gb2, gW3T, gb3;
  DevBuf<double> partial;
  void alloc(Ctx& c, const MlpNet& net, int B_) {
    B = B_;
    X.alloc(c, static_cast<size_t>(B) * net.dp);
    XT.alloc(c, static_cast<size_t>(B) * net.dp);
    H1.alloc(c, static_cast<size_t>(B) * MLP_H);
    H1T.alloc(c, static_cast<size_t>(B) * MLP_H);
    H2.alloc(c, static_cast<size_t>(B) * MLP_H);
    H2T.alloc(c, static_cast<size_t>(B) * MLP_H);
    dZ3.alloc(c, static_cast<size_t>(B) * net.dp64);
    dZ3T.alloc(c, static_cast<size_t>(B) * net.dp16);
    dZ2.alloc(c, static_cast<size_t>(B) * MLP_H);
    dZ2T.alloc(c, static_cast<size_t>(B) * MLP_H);
    dZ1.alloc(c, static_cast<size_t>(B) * MLP_H);
    dZ1T.alloc(c, static_cast<size_t>(B) * MLP_H);
    out.alloc(c, static_cast<size_t>(B) * net.dp16);
    tgt.alloc(c, static_cast<size_t>(B) * net.dim);
    gW1.alloc(c, net.W1.count);
    gb1.alloc(c, MLP_H);
    gW2.alloc(c, net.W2.count);
    gb2.alloc(c, MLP_H);
    gW3T.alloc(c, net.W3T.count);
    gb3.alloc(c, net.dp16);
    partial.alloc(c, 64);
  }
};

// Forward + backward of one batch (X and tgt already filled); gradients into bt.g*, returns nothing
// (the loss partials are in bt.partial).
void mlp_forward_backward(Ctx& c, MlpNet& net, MlpBatch& bt) {
  const int B = bt.B;
  mlp_forward(c, net, bt.X.get(), B, bt.H1.get(), bt.H2.get(), bt.out.get(), B);
  mse_grad_kernel<<<64, 256, 0, c.stream>>>(bt.out.get(), net.dp16, bt.tgt.get(), B, net.dim, net.dp64, bt.dZ3.get(),
                                           bt.partial.get());
  PM_LAUNCHED();
  // dW3^T [512][dp16] = H2^T . dZ3  (A = H2^T [512][B], B = dZ3^T [dp16][B], K = B)
  transpose(c, bt.H2.get(), B, MLP_H, bt.H2T.get());
  // dZ3^T [dp16][B]: transpose [B][dp64] into scratch [dp64][B] (dZ1T has room), keep its first dp16 rows
  transpose(c, bt.dZ3.get(), B, net.dp64, bt.dZ1T.get());
  PM_CUDA(cudaMemcpyAsync(bt.dZ3T.get(), bt.dZ1T.get(), static_cast<size_t>(net.dp16) * B * 2, cudaMemcpyDeviceToDevice,
                          c.stream));
  GemmOut g3{};
  g3.out_f32 = bt.gW3T.get();
  g3.ld_out = net.dp16;
  g3.m_valid = MLP_H;
  g3.n_valid = net.dp16;
  gemm<16, EPI_F32>(c, bt.H2T.get(), MLP_H, bt.dZ3T.get(), net.dp16, B, g3);
  colsum_bf16_kernel<<<1, 64, 0, c.stream>>>(bt.dZ3.get(), B, net.dp16, net.dp64, bt.gb3.get());
  PM_LAUNCHED();
  // dZ2 = (dZ3 . W3) * relu'(H2): A = dZ3 [B][dp64], B = W3Tb [512][dp64], K = dp64
  GemmOut g2{};
  g2.out_bf16 = bt.dZ2.get();
  g2.aux = bt.H2.get();
  g2.ld_out = MLP_H;
  g2.ld_aux = MLP_H;
  g2.m_valid = B;
  g2.n_valid = MLP_H;
  gemm<128, EPI_DRELU>(c, bt.dZ3.get(), B, net.W3Tb.get(), MLP_H, net.dp64, g2);
  // dW2 [512][512] = dZ2^T . H1 (A = dZ2^T [512][B], B = H1^T [512][B], K = B)
  transpose(c, bt.dZ2.get(), B, MLP_H, bt.dZ2T.get());
  transpose(c, bt.H1.get(), B, MLP_H, bt.H1T.get());
  GemmOut w2{};
  w2.out_f32 = bt.gW2.get();
  w2.ld_out = MLP_H;
  w2.m_valid = MLP_H;
  w2.n_valid = MLP_H;
  gemm<128, EPI_F32>(c, bt.dZ2T.get(), MLP_H, bt.H1T.get(), MLP_H, B, w2);
  colsum_bf16_kernel<<<ceil_div(MLP_H, 128), 128, 0, c.stream>>>(bt.dZ2.get(), B, MLP_H, MLP_H, bt.gb2.get());
  PM_LAUNCHED();
  // dZ1 = (dZ2 . W2) * relu'(H1): A = dZ2 [B][512], B = W2^T [512][512], K = 512
  GemmOut g1{};
  g1.out_bf16 = bt.dZ1.get();
  g1.aux = bt.H1.get();
  g1.ld_out = MLP_H;
  g1.ld_aux = MLP_H;
  g1.m_valid = B;
  g1.n_valid = MLP_H;
  gemm<128, EPI_DRELU>(c, bt.dZ2.get(), B, net.W2Tb.get(), MLP_H, MLP_H, g1);
  // dW1 [512][dp] = dZ1^T . X (A = dZ1^T [512][B], B = X^T [dp][B], K = B)
  transpose(c, bt.dZ1.get(), B, MLP_H, bt.dZ1T.get());
  transpose(c, bt.X.get(), B, net.dp, bt.XT.get());
  GemmOut w1{};
  w1.out_f32 = bt.gW1.get();
  w1.ld_out = net.dp;
  w1.m_valid = MLP_H;
  w1.n_valid = net.dp;
  if (net.dp % 128 == 0)
    gemm<128, EPI_F32>(c, bt.dZ1T.get(), MLP_H, bt.XT.get(), net.dp, B, w1);
  else
    gemm<64, EPI_F32>(c, bt.dZ1T.get(), MLP_H, bt.XT.get(), net.dp, B, w1);
  colsum_bf16_kernel<<<ceil_div(MLP_H, 128), 128, 0, c.stream>>>(bt.dZ1.get(), B, MLP_H, MLP_H, bt.gb1.get());
  PM_LAUNCHED();
}

void adamw_step(Ctx& c, MlpNet& net, MlpBatch& bt, std::vector<DevBuf<float>>& mom, float lr, float wd, int t) {
  const float b1c = 1.0f - std::pow(0.9f, static_cast<float>(t));
  const float b2c = 1.0f - std::pow(0.999f, static_cast<float>(t));
  float* P[6] = {net.W1.get(), net.b1.get(), net.W2.get(), net.b2.get(), net.W3T.get(), net.b3.get()};
  float* G[6] = {bt.gW1.get(), bt.gb1.get(), bt.gW2.get(), bt.gb2.get(), bt.gW3T.get(), bt.gb3.get()};
  const uint64_t N[6] = {net.W1.count, net.b1.count, net.W2.count, net.b2.count, net.W3T.count, net.b3.count};
  for (int q = 0; q < 6; ++q) {
    const float decay = (q % 2 == 0) ? wd : 0.0f;  // weights decay, biases do not
    adamw_kernel<<<static_cast<unsigned>(std::min<uint64_t>(ceil_div(N[q], 256), 1024)), 256, 0, c.stream>>>(
        P[q], G[q], mom[2 * q].get(), mom[2 * q + 1].get(), N[q], lr, decay, b1c, b2c, nullptr);
    PM_LAUNCHED();
  }
  net.refresh(c);
}

}  // namespace

uint64_t mlp_param_count(uint64_t d, uint64_t dim) {
  return static_cast<uint64_t>(MLP_H) * d + MLP_H + static_cast<uint64_t>(MLP_H) * MLP_H + MLP_H + dim * MLP_H + dim;
}

void mlp_init_params(uint64_t d, uint64_t dim, uint64_t seed, float* flat) {
  // PyTorch-style default: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases, seeded.
  std::mt19937_64 rng(seed);
  auto fill = [&](float* p, uint64_t cnt, double fan_in) {
    std::uniform_real_distribution<double> u(-1.0 / std::sqrt(fan_in), 1.0 / std::sqrt(fan_in));
    for (uint64_t i = 0; i < cnt; ++i) p[i] = static_cast<float>(u(rng));
  };
  float* p = flat;
  fill(p, MLP_H * d, static_cast<double>(d));
  p += MLP_H * d;
  fill(p, MLP_H, static_cast<double>(d));
  p += MLP_H;
  fill(p, static_cast<uint64_t>(MLP_H) * MLP_H, MLP_H);
  p += static_cast<uint64_t>(MLP_H) * MLP_H;
  fill(p, MLP_H, MLP_H);
  p += MLP_H;
  fill(p, dim * MLP_H, MLP_H);
  p += dim * MLP_H;
  fill(p, dim, MLP_H);
}

void mlp_apply_device(Ctx& c, const float* params, uint64_t d, uint64_t dim, const float* d_x, uint64_t n,
                      float* d_out) {
  PM_REQUIRE(d >= 1 && d <= 4096 && dim >= 1 && dim <= 16, PACMAP_ERR_UNSUPPORTED, "MLP supports d <= 4096, dim <= 16");
  MlpNet net;
  net.alloc(c, static_cast<int>(d), static_cast<int>(dim));
  net.upload(c, params);
  const uint64_t chunk = 1ull << 20;  // rows per pass (bounded scratch: 2.3 GB at d = 128)
  DevBuf<__nv_bfloat16> X(c, chunk * net.dp), H1(c, chunk * MLP_H), H2(c, chunk * MLP_H);
  DevBuf<float> out(c, chunk * net.dp16);
  for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
    const uint64_t rows = std::min<uint64_t>(chunk, n - r0);
    const int rows_pad = pad_to(static_cast<int>(rows), 128);
    cast_pad(c, d_x + r0 * d, nullptr, rows, static_cast<int>(d), static_cast<int>(d), rows_pad, net.dp, X.get());
    mlp_forward(c, net, X.get(), rows_pad, H1.get(), H2.get(), out.get(), static_cast<int>(rows));
    PM_CUDA(cudaMemcpy2DAsync(d_out + r0 * dim, dim * 4, out.get(), net.dp16 * 4, dim * 4, rows,
                              cudaMemcpyDeviceToDevice, c.stream));
  }
  c.check_errors("MLP inference");
}

void mlp_grad_device(Ctx& c, const float* params, uint64_t d, uint64_t dim, const float* d_x, const float* d_t,
                     uint64_t B, float* grads_flat, float* loss) {
  PM_REQUIRE(B % 128 == 0 && B > 0, PACMAP_ERR_UNSUPPORTED, "MLP batch must be a positive multiple of 128");
  MlpNet net;
  net.alloc(c, static_cast<int>(d), static_cast<int>(dim));
  net.upload(c, params);
  MlpBatch bt;
  bt.alloc(c, net, static_cast<int>(B));
  cast_pad(c, d_x, nullptr, B, static_cast<int>(d), static_cast<int>(d), B, net.dp, bt.X.get());
  PM_CUDA(cudaMemcpyAsync(bt.tgt.get(), d_t, B * dim * 4, cudaMemcpyDeviceToDevice, c.stream));
  mlp_forward_backward(c, net, bt);
  // gradients into the flat layout (reuse the download path through a scratch network)
  MlpNet g;
  g.alloc(c, static_cast<int>(d), static_cast<int>(dim));
  PM_CUDA(cudaMemcpyAsync(g.W1.get(), bt.gW1.get(), bt.gW1.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  PM_CUDA(cudaMemcpyAsync(g.b1.get(), bt.gb1.get(), bt.gb1.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  PM_CUDA(cudaMemcpyAsync(g.W2.get(), bt.gW2.get(), bt.gW2.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  PM_CUDA(cudaMemcpyAsync(g.b2.get(), bt.gb2.get(), bt.gb2.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  PM_CUDA(cudaMemcpyAsync(g.W3T.get(), bt.gW3T.get(), bt.gW3T.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  PM_CUDA(cudaMemcpyAsync(g.b3.get(), bt.gb3.get(), bt.gb3.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  g.download(c, grads_flat);
  std::vector<double> part(64);
  PM_CUDA(cudaMemcpyAsync(part.data(), bt.partial.get(), 64 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  PM_CUDA(cudaStreamSynchronize(c.stream));
  double s = 0.0;
  for (double v : part) s += v;
  *loss = static_cast<float>(s / static_cast<double>(B * dim));
  c.check_errors("MLP gradient");
}

void mlp_train_device(Ctx& c, float* params, uint64_t d, uint64_t dim, const float* d_x, const float* d_t,
                      uint64_t n, uint64_t epochs, uint64_t batch, float lr, float wd, uint64_t seed,
                      float* epoch_loss) {
  PM_REQUIRE(batch % 128 == 0 && batch > 0 && batch <= n, PACMAP_ERR_UNSUPPORTED,
             "MLP batch must be a positive multiple of 128 and at most n");
  MlpNet net;
  net.alloc(c, static_cast<int>(d), static_cast<int>(dim));
  net.upload(c, params);
  MlpBatch bt;
  bt.alloc(c, net, static_cast<int>(batch));
  std::vector<DevBuf<float>> mom(12);
  const uint64_t cnt[6] = {net.W1.count, net.b1.count, net.W2.count, net.b2.count, net.W3T.count, net.b3.count};
  for (int q = 0; q < 6; ++q) {
    mom[2 * q].alloc(c, cnt[q]);
    mom[2 * q + 1].alloc(c, cnt[q]);
    PM_CUDA(cudaMemsetAsync(mom[2 * q].get(), 0, cnt[q] * 4, c.stream));
    PM_CUDA(cudaMemsetAsync(mom[2 * q + 1].get(), 0, cnt[q] * 4, c.stream));
  }
  std::vector<uint32_t> perm(n);
  DevBuf<uint32_t> dperm(c, n);
  std::mt19937_64 rng(seed);
  const uint64_t steps = n / batch;
  int t = 0;
  for (uint64_t ep = 0; ep < epochs; ++ep) {
    for (uint64_t i = 0; i < n; ++i) perm[i] = static_cast<uint32_t>(i);
    std::shuffle(perm.begin(), perm.end(), rng);
    PM_CUDA(cudaMemcpyAsync(dperm.get(), perm.data(), n * 4, cudaMemcpyHostToDevice, c.stream));
    double ep_loss = 0.0;
    for (uint64_t st = 0; st < steps; ++st) {
      const uint32_t* rows = dperm.get() + st * batch;
      cast_pad(c, d_x, rows, batch, static_cast<int>(d), static_cast<int>(d), batch, net.dp, bt.X.get());
      // targets gathered through the same rows
      gather_rows_kernel<<<ceil_div(batch * dim, 256), 256, 0, c.stream>>>(d_t, rows, batch, static_cast<int>(dim),
                                                                          bt.tgt.get());
      PM_LAUNCHED();
      mlp_forward_backward(c, net, bt);
      adamw_step(c, net, bt, mom, lr, wd, ++t);
      std::vector<double> part(64);
      PM_CUDA(cudaMemcpyAsync(part.data(), bt.partial.get(), 64 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
      PM_CUDA(cudaStreamSynchronize(c.stream));
      double s = 0.0;
      for (double v : part) s += v;
      ep_loss += s / static_cast<double>(batch * dim);
    }
    if (epoch_loss) epoch_loss[ep] = static_cast<float>(ep_loss / std::max<uint64_t>(steps, 1));
  }
  c.check_errors("MLP training");
  net.download(c, params);
}

}  // namespace pacmap
