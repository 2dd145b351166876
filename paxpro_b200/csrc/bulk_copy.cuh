// bulk_copy.cuh -- TMA bulk copies (cp.async.bulk) between global and shared
// memory, with an mbarrier for the loads and bulk groups for the stores.
//
// A load is issued by any thread and counted on the CTA's mbarrier in bytes
// (complete_tx); one thread arms the barrier with the total byte count
// (arrive.expect_tx) before any copy is issued.  Stores read shared memory
// through the async proxy: writers fence (fence.proxy.async.shared::cta)
// before the CTA barrier that precedes the stores, and each issuing thread
// waits for its stores to have read shared memory before the CTA exits.
// Addresses: 16-byte aligned at both ends, sizes multiples of 16 bytes.  No
// copy here uses cluster multicast.
#pragma once
#include <cstdint>

namespace pxp {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Arrive once and add `bytes` to the transaction count of the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Wait for the phase with the given parity to complete, giving up after
// about `limit_ns` of global time (and at most 2^26 polls).  Returns whether
// the phase completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                  unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0; it < (1u << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0 && global_ns() - t0 > limit_ns) break;
  }
  return false;
}

// global -> shared, counted on `bar`.
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src, unsigned bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst_smem)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// shared -> global, in this thread's current bulk group.
__device__ __forceinline__ void bulk_store(void *dst, const void *src_smem, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst),
               "r"(smem_u32(src_smem)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }

// Wait until this thread's committed bulk stores have read shared memory.
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}

// Make this thread's generic-proxy shared-memory writes visible to the async
// proxy (bulk stores issued after the next CTA barrier).
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

}  // namespace pxp
