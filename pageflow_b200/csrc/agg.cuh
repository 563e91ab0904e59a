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

// Hot-group combining without a full match: each step tries a few candidate
// groups - the warp's hot group from the step before, then the group of the
// first lane not yet served - and the lanes holding a candidate (two or more
// of them) add their values with one warp reduction and one atomic pair; the
// other lanes issue their own atomic pair.  Exact (every lane's value is
// added once), a few ballots a step for distinct groups, and a step of hot
// keys costs about one atomic pair a candidate.  hot is the warp's state
// (read from its first active lane).
#ifndef PF_HOT_ROUNDS
#define PF_HOT_ROUNDS 2
#endif

__device__ __forceinline__ void hot_add(unsigned long long* slab, long long g, long long value,
                                        long long& hot) {
  const unsigned act = __activemask();
  const int lane = threadIdx.x & 31;
  unsigned todo = __ballot_sync(act, g >= 0);  // lanes not served yet
  unsigned untried = todo;                      // lanes whose group was no candidate
  long long next_hot = hot;
  int best = 1;
#pragma unroll
  for (int r = 0; r < PF_HOT_ROUNDS; ++r) {
    if (r > 0 && !untried) break;
    // one candidate for the whole warp: lanes that reached an earlier step
    // apart (independent thread scheduling) may hold different hot groups
    const long long c = __shfl_sync(act, r == 0 ? hot : g, r == 0 ? __ffs(act) - 1
                                                                  : __ffs(untried) - 1);
    const unsigned m = __ballot_sync(act, g == c) & todo;
    untried &= ~m;
    const int n = __popc(m);
    if (n >= 2) {
      if ((m >> lane) & 1u) {
        const unsigned long long v = (unsigned long long)value;
        const unsigned s0 = __reduce_add_sync(m, (unsigned)(v & 0x3fffff));
        const unsigned s1 = __reduce_add_sync(m, (unsigned)((v >> 22) & 0x3fffff));
        const unsigned s2 = __reduce_add_sync(m, (unsigned)(v >> 44));
        if (lane == __ffs(m) - 1) {
          const unsigned long long sum = (unsigned long long)s0 +
                                         ((unsigned long long)s1 << 22) +
                                         ((unsigned long long)s2 << 44);
          atomicAdd(&slab[2 * (unsigned long long)c], sum);
          atomicAdd(&slab[2 * (unsigned long long)c + 1], (unsigned long long)n);
        }
      }
      todo &= ~m;
      if (n > best) {
        best = n;
        next_hot = c;
      }
    } else if (r > 0 && best < 2) {
      next_hot = c;  // nothing repeated yet: try this group first next step
    }
  }
  if ((todo >> lane) & 1u) {
    atomicAdd(&slab[2 * (unsigned long long)g], (unsigned long long)value);
    atomicAdd(&slab[2 * (unsigned long long)g + 1], 1ULL);
  }
  hot = next_hot;
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

// A block's group cache in shared memory: CACHE_SLOTS groups, direct-mapped
// by a multiplicative hash of the group; a thread adds (sum, count) into its
// group's slot when the slot holds that group or is free (claimed by a CAS),
// and into the global slab otherwise.  cache_flush moves every cached group
// into the slab and empties the cache (every thread of the block calls it).
// Hot groups of skewed data then cost one global atomic pair a block and
// flush; distinct groups cost about what direct atomics do.
#ifndef PF_CACHE_LOG
#define PF_CACHE_LOG 10
#endif
constexpr int CACHE_SLOTS = 1 << PF_CACHE_LOG;
constexpr long long CACHE_EMPTY = -1;

// A slot's sum is two 32-bit words (the low word's add returns its old value,
// which shows the carry into the high word) and its count one: 64-bit adds on
// shared memory cost far more than 32-bit ones, and a slot's count between
// two flushes (one work item's rows) stays below 2^32.
struct GroupCache {
  long long tag[CACHE_SLOTS];
  unsigned lo[CACHE_SLOTS];
  unsigned hi[CACHE_SLOTS];
  unsigned cnt[CACHE_SLOTS];
};

__device__ __forceinline__ void cache_init(GroupCache& gc) {
  for (int i = threadIdx.x; i < CACHE_SLOTS; i += blockDim.x) {
    gc.tag[i] = CACHE_EMPTY;
    gc.lo[i] = 0;
    gc.hi[i] = 0;
    gc.cnt[i] = 0;
  }
}

__device__ __forceinline__ void cache_add(GroupCache& gc, unsigned long long* slab, long long g,
                                          unsigned long long sum, unsigned long long cnt) {
  const unsigned slot = ((unsigned)g * 0x9E3779B1u) >> (32 - PF_CACHE_LOG);
  long long t = *(volatile long long*)&gc.tag[slot];
  if (t == CACHE_EMPTY) {
    const long long old = (long long)atomicCAS((unsigned long long*)&gc.tag[slot],
                                               (unsigned long long)CACHE_EMPTY,
                                               (unsigned long long)g);
    t = old == CACHE_EMPTY ? g : old;
  }
  if (t == g) {
    const unsigned l = (unsigned)sum, h = (unsigned)(sum >> 32);
    const unsigned old = atomicAdd(&gc.lo[slot], l);
    const unsigned hc = h + (old + l < old ? 1u : 0u);
    if (hc) atomicAdd(&gc.hi[slot], hc);
    atomicAdd(&gc.cnt[slot], (unsigned)cnt);
  } else {
    atomicAdd(&slab[2 * (unsigned long long)g], sum);
    atomicAdd(&slab[2 * (unsigned long long)g + 1], cnt);
  }
}

__device__ __forceinline__ void cache_flush(GroupCache& gc, unsigned long long* slab) {
  __syncthreads();
  for (int i = threadIdx.x; i < CACHE_SLOTS; i += blockDim.x) {
    const long long g = gc.tag[i];
    if (g != CACHE_EMPTY) {
      atomicAdd(&slab[2 * (unsigned long long)g],
                ((unsigned long long)gc.hi[i] << 32) | gc.lo[i]);
      atomicAdd(&slab[2 * (unsigned long long)g + 1], (unsigned long long)gc.cnt[i]);
      gc.tag[i] = CACHE_EMPTY;
      gc.lo[i] = 0;
      gc.hi[i] = 0;
      gc.cnt[i] = 0;
    }
  }
  __syncthreads();
}

}  // namespace pf
