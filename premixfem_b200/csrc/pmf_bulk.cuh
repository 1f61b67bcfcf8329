// Bulk (TMA-engine) copies from global into shared memory, completed on an
// mbarrier, for the subdomain kernels that stage a contiguous block of
// per-subdomain data (the level-1 IC(0) factor, the local eigensolver's sweep
// coefficients).  Plain per-CTA copies: no cluster multicast.
#pragma once
#include <stdint.h>

namespace pmf {

constexpr long long kBulkSpinLimit = 1LL << 22;  // mbarrier polls before a CTA gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// global -> shared bulk copy; bytes a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Thread 0's bounded wait for phase 0 of the mbarrier.  Returns false if the
// copy did not land within kBulkSpinLimit polls; it then waits once more
// (bounded) so that a late copy does not land in shared memory after the CTA
// has moved on.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b) {
  long long spins = 0;
  while (!mbar_try_wait(b, 0))
    if (++spins > kBulkSpinLimit) {
      for (long long s2 = 0; s2 < kBulkSpinLimit && !mbar_try_wait(b, 0); ++s2) {
      }
      return false;
    }
  return true;
}

}  // namespace pmf
