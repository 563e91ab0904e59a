// Device helpers shared by the persistent kernels (batch.cu, serve.cu): an
// acquire load for their bounded waits, and the warp-combined (sum, count)
// update of a group slab.
#pragma once

#include "common.cuh"

// 1: a persistent kernel's block takes its next work item while it works on
// the current one; 0: when it is done with it.
#ifndef PF_PREFETCH_ITEMS
#define PF_PREFETCH_ITEMS 0
#endif
// adaptive_add's mode: 1 combine equal groups in a warp before the atomics
// always; 0: one atomic pair a row; 2: adaptive (see Combiner).
#ifndef PF_COMBINE
#define PF_COMBINE 2
#endif

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

// Adaptive combining: a warp combines while combining pays (it saved at least
// COMBINE_MIN atomic pairs in the warp's last combined step), and otherwise
// issues one atomic pair a row, checking again every COMBINE_RECHECK steps.
// Uniform groups skip the match; hot groups (few groups, skewed keys) are
// combined.  Every lane of the warp holds the same state.
constexpr int COMBINE_MIN = 4;
constexpr int COMBINE_RECHECK = 16;

struct Combiner {
  int left = 0;  // plain steps before the next check (0: combine now)
};

__device__ __forceinline__ void adaptive_add(unsigned long long* slab, long long g,
                                             long long value, Combiner& c) {
  if (PF_COMBINE == 0 || (PF_COMBINE == 2 && c.left > 0)) {
    if (g >= 0) {
      atomicAdd(&slab[2 * (unsigned long long)g], (unsigned long long)value);
      atomicAdd(&slab[2 * (unsigned long long)g + 1], 1ULL);
    }
    --c.left;
    return;
  }
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, g);
  const int lane = threadIdx.x & 31;
  const bool leader = lane == __ffs(peers) - 1;
  if (PF_COMBINE == 2) {
    const unsigned valid = __ballot_sync(act, g >= 0);
    const unsigned leaders = __ballot_sync(act, g >= 0 && leader);
    c.left = __popc(valid) - __popc(leaders) >= COMBINE_MIN ? 0 : COMBINE_RECHECK;
  }
  if (g < 0) return;
  const unsigned long long v = (unsigned long long)value;
  const unsigned s0 = __reduce_add_sync(peers, (unsigned)(v & 0x3fffff));
  const unsigned s1 = __reduce_add_sync(peers, (unsigned)((v >> 22) & 0x3fffff));
  const unsigned s2 = __reduce_add_sync(peers, (unsigned)(v >> 44));
  if (leader) {
    const unsigned long long sum =
        (unsigned long long)s0 + ((unsigned long long)s1 << 22) + ((unsigned long long)s2 << 44);
    atomicAdd(&slab[2 * (unsigned long long)g], sum);
    atomicAdd(&slab[2 * (unsigned long long)g + 1], (unsigned long long)__popc(peers));
  }
}

}  // namespace pf
