// Inline-PTX helpers shared by the sm_100a kernels: mbarriers (bounded waits), bulk copies.
#pragma once
#include <cstdint>

namespace pacmap {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// *p = (a, b) when x >= y, as one predicated store (no branch, nothing written otherwise); returns 1 when
// it stored, else 0 (the same predicate, not a second comparison).
__device__ __forceinline__ uint32_t st_global_v2_if_ge(void* p, uint32_t a, uint32_t b, float x, float y) {
  uint32_t stored;
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ge.f32 q, %4, %5;\n\t@q st.global.v2.u32 [%1], {%2, %3};\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(stored)
      : "l"(p), "r"(a), "r"(b), "f"(x), "f"(y)
      : "memory");
  return stored;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s: far above any legitimate wait in this library

// Bounded wait on a barrier phase: false when it gave up (timeout, or *abort_flag became non-zero).
__device__ __noinline__ inline bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (globaltimer() - t0 > WAIT_LIMIT_NS) return false;
    }
  }
}

// Untiled bulk copy global -> shared (both 16-byte aligned, size a multiple of 16), completing on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

}  // namespace pacmap
