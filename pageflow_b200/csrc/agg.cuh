// Device helpers shared by the persistent kernels (batch.cu, serve.cu): an
// acquire load for their bounded waits, and the warp-combined (sum, count)
// update of a group slab.
#pragma once

#include "common.cuh"

namespace pf {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Warp-combined RED of (value, 1) into group g's pair (g < 0: none): lanes
// holding the same group add their values (exactly, in three 22-bit slices of
// the 64-bit two's-complement word) and one lane issues the atomics.
__device__ __forceinline__ void combined_add(unsigned long long* slab, long long g,
                                             long long value) {
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, g);
  if (g < 0) return;
  const unsigned long long v = (unsigned long long)value;
  const unsigned s0 = __reduce_add_sync(peers, (unsigned)(v & 0x3fffff));
  const unsigned s1 = __reduce_add_sync(peers, (unsigned)((v >> 22) & 0x3fffff));
  const unsigned s2 = __reduce_add_sync(peers, (unsigned)(v >> 44));
  const int lane = threadIdx.x & 31;
  if (lane == __ffs(peers) - 1) {
    const unsigned long long sum =
        (unsigned long long)s0 + ((unsigned long long)s1 << 22) + ((unsigned long long)s2 << 44);
    atomicAdd(&slab[2 * (unsigned long long)g], sum);
    atomicAdd(&slab[2 * (unsigned long long)g + 1], (unsigned long long)__popc(peers));
  }
}

}  // namespace pf
