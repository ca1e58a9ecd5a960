// Bulk copies global -> shared memory (cp.async.bulk, the copy engine of
// sm_90+ that TMA also uses, here in its untiled form) with completion counted
// on an mbarrier in shared memory, and bounded waits on that mbarrier.
//
// A copy starts at a 16-byte aligned global address, lands at a 16-byte
// aligned shared address and moves a multiple of 16 bytes; every caller in
// this library checks that on the host (layout strides) or by construction.
// A wait polls mbarrier.try_wait a bounded number of times and reports
// whether the phase completed; callers record a fault and stop instead of
// spinning forever.
#pragma once

namespace gsb {

constexpr unsigned kBulkSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// One arrival per phase (the producer's arrive.expect_tx); the fence makes
// the initialised barrier visible to the copy engine.
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy; addresses 16-byte aligned, size a multiple of 16
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy ones (a bulk copy refilling a buffer just read).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `bar` with the given parity; false when it
// gave up.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity = 0) {
  for (unsigned spins = 0; spins < kBulkSpinLimit; ++spins)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace gsb
