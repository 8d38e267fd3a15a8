// bulk.cuh -- mbarrier + cp.async.bulk (1-D TMA) staging helpers, sm_90+/sm_100a.
//
// Every wait is bounded: a try_wait loop gives up after kWaitNs nanoseconds
// of %globaltimer (or kSpinLimit polls) and reports failure to the caller,
// which records an error status and stops instead of hanging the GPU.
#pragma once
#include <stdint.h>

namespace art {

constexpr uint32_t kSpinLimit = 1u << 26;
constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; returns false if the barrier did not complete in time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 63u && globaltimer_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

// 1-D bulk copy global -> shared, completion counted on `bar` (bytes).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// A byte range [src, src+bytes) widened to whole 16-byte granules.  Reading
// a whole granule never leaves the page of its first valid byte, so the
// widening is always mapped memory.
struct Granules {
  const char* base;   // 16-byte aligned start
  uint32_t lead;      // bytes skipped at the front (src - base)
  uint32_t bytes;     // multiple of 16
};
__device__ __forceinline__ Granules granules(const void* src, uint64_t nbytes) {
  uintptr_t s = (uintptr_t)src;
  uintptr_t b = s & ~(uintptr_t)15;
  uintptr_t e = (s + nbytes + 15) & ~(uintptr_t)15;
  Granules g;
  g.base = (const char*)b;
  g.lead = (uint32_t)(s - b);
  g.bytes = (uint32_t)(e - b);
  if (nbytes == 0) g.bytes = 0;
  return g;
}

}  // namespace art
