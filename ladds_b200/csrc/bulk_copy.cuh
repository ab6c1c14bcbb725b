// bulk_copy.cuh -- one-dimensional bulk copies global -> shared memory by the
// tensor memory accelerator (cp.async.bulk, sm_90 and later), completed on a
// shared-memory mbarrier, and a bounded wait for them.
//
// Rules the callers keep: source and destination addresses 16-byte aligned,
// sizes multiples of 16 bytes; the expected transaction bytes of a phase equal
// the bytes of the copies issued for it; no copy is left in flight when the
// CTA exits (every issued phase is waited for).  No multicast form is used:
// every copy reads this GPU's own memory into its own CTA.
#pragma once
#include <cstdint>

namespace ladds {

__device__ __forceinline__ uint32_t smemAddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// one thread: an mbarrier expecting `count` arrivals per phase
__device__ __forceinline__ void mbarInit(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the async proxy (before the CTA barrier that follows)
__device__ __forceinline__ void mbarInitFence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's earlier shared-memory accesses before later async-proxy
// writes to the same memory (a buffer the CTA has read is refilled)
__device__ __forceinline__ void asyncProxyFence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// arrives on the barrier and adds `bytes` to the transactions its phase waits for
__device__ __forceinline__ void mbarArriveExpectTx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
               : "memory");
}

// bytes (multiple of 16) from global src to shared dst, both 16-byte aligned;
// completion counted on bar
__device__ __forceinline__ void bulkLoad(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smemAddr(dst)),
      "l"(src), "r"(bytes), "r"(smemAddr(bar))
      : "memory");
}

// waits until the barrier's phase with the given parity has completed, at most
// `limit` polls; false if it has not (the caller reports it and goes on)
__device__ __forceinline__ bool mbarWait(unsigned long long *bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smemAddr(bar);
  for (uint32_t k = 0; k < limit; ++k) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace ladds
