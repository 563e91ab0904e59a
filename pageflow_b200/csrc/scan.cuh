// Ordered stream compaction and int64 scans shared by the join cores and the
// slab: block counts, a scan of the block counts, then each block writes its
// kept items at its offset, in row order.
#pragma once

#include "common.cuh"

namespace pf {

constexpr int CT = 256;          // threads of a compaction block
constexpr int CITEMS = 16;       // rows a thread
constexpr int CB = CT * CITEMS;  // rows a compaction block covers
static_assert(CB <= 65536, "block-local rows are 16-bit");

// Exclusive scan in place of n int64 values by one block of 1024 threads;
// the total goes to *total (device) and, when host is not null, to *host.
__global__ void k_scan_counts(long long* __restrict__ a, long long n, long long* total,
                              long long* host);

// dst[i] = src[i] for i < n (one block; dst may be a pinned buffer's alias).
__global__ void k_copy_i64(const long long* src, long long* dst, long long n);

// Device-wide scan of n int64 values (in -> out, inclusive or exclusive),
// the total into *total (device).  Scratch: scan_scratch_elems(n) int64.
int64_t scan_scratch_elems(int64_t n);
int scan_i64(const long long* in, long long* out, long long n, bool inclusive, long long* total,
             long long* scratch, cudaStream_t st);

// Within a block of CT threads: each thread's CITEMS flags (row order: thread
// t holds rows t*CITEMS .. t*CITEMS+CITEMS-1) -> each kept row's rank in the
// block, and the block's total.  One __syncthreads pair.
__device__ __forceinline__ int block_ranks(const bool (&keep)[CITEMS], int (&rank)[CITEMS],
                                           int* wsum /* [CT/32] smem */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int c = 0;
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) c += keep[k];
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  int pre = 0, tot = 0;
#pragma unroll
  for (int q = 0; q < CT / 32; ++q) {
    const int t = wsum[q];
    pre += q < w ? t : 0;
    tot += t;
  }
  int r = pre + incl - c;
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) {
    rank[k] = r;
    r += keep[k];
  }
  __syncthreads();
  return tot;
}

// block_ranks, then each kept row's block-local index (t*CITEMS + k) staged
// at its rank in rows[] (shared memory, CB entries), so that the block writes
// its kept rows out with consecutive threads on consecutive outputs.  Returns
// the block's total; rows[] is complete on return.
__device__ __forceinline__ int block_compact(const bool (&keep)[CITEMS], int (&rank)[CITEMS],
                                             unsigned short* rows, int* wsum) {
  const int tot = block_ranks(keep, rank, wsum);
#pragma unroll
  for (int k = 0; k < CITEMS; ++k)
    if (keep[k]) rows[rank[k]] = (unsigned short)(threadIdx.x * CITEMS + k);
  __syncthreads();
  return tot;
}

}  // namespace pf
