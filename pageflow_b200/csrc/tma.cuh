// Bulk asynchronous copies (the TMA engine's non-tensor form) from global to
// shared memory, completed on an mbarrier, for sm_100a.  Copies are per-CTA:
// no cluster multicast is ever issued.  Every wait is bounded: a wait that
// runs out reports false and the caller takes its error path.
#pragma once

#include <stdint.h>

namespace pf {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes initialised mbarriers visible to the async proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also expects `bytes` of transaction completions.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// dst (shared, 16-byte aligned) <- src (global, 16-byte aligned), bytes a
// multiple of 16; completes `bytes` transactions on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Asks the TMA engine to bring [p, p + bytes) of global memory into L2 (no
// destination, nothing to wait for).  Only whole 16-byte units inside the
// range are named: the start is rounded up and the end down, so nothing
// outside it is touched; pieces of at most 64 KiB.
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned long long bytes) {
  unsigned long long a = ((unsigned long long)p + 15) & ~15ULL;
  const unsigned long long e = ((unsigned long long)p + bytes) & ~15ULL;
  for (; a < e; a += 65536) {
    const unsigned n = (unsigned)(e - a < 65536 ? e - a : 65536);
    asm volatile(
        "{\n .reg .u64 g;\n cvta.to.global.u64 g, %0;\n"
        " cp.async.bulk.prefetch.L2.global [g], %1;\n}" ::"l"(a),
        "r"(n)
        : "memory");
  }
}

// dst (global, 16-byte aligned) <- src (shared, 16-byte aligned), bytes a
// multiple of 16, in this thread's current bulk group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Until this thread's committed bulk copies have read their shared-memory
// sources (the hardware's own wait: no spin).
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Until this thread's committed bulk copies are complete.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of `parity` to complete, at most `limit` polls (each
// poll itself suspends the thread for a bounded time); false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  unsigned limit = 1u << 24) {
  for (unsigned i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace pf
