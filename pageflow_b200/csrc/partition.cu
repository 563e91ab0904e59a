// Stable radix partition into PageFlow's padded bucket layout: the sm_100a
// replacement of tqpkernels.partition_sort (reference
// operators/kernels/partition_sort.cu:610-768, wrapper
// operators/partition_sort.py:68-143).
//
// Work split.  The domain (the pre-mask rows, or the kept rows after the
// select-first prologue) is cut into CHUNKS of one 2048-row sub-tile (more
// only when the chunk histograms would pass 2^24 entries).  Every chunk owns
// a single run of every bucket, at an offset the chunk histograms fix, which
// keeps the partition stable; the scatter runs one CTA a chunk, so the chunks
// at work at one time are neighbours:
//
//   k_hist      one histogram row per chunk, hist[chunk][b] (coalesced)
//   k_scan      per bucket, exclusive offsets over the chunks (k_scan_sum,
//               k_scan_groups, k_scan_write: the chunks in 64 groups, each
//               group's sums, a scan over the groups, the offsets)
//   k_bases     bucket counts, each row-width class's padded bucket starts and
//               total, all written into the caller's pinned host_out through
//               its device alias; an overflow check against n_valid
//   k_scatter   per sub-tile: warp-match ranks (stable), the sub-tile's bucket
//               runs, the rows staged in shared memory in bucket order, every
//               column and the gidx written as coalesced bucket runs
//
// Mask prologues (same chunking as the main walk):
//   compacted-input  k_mask_count + k_scan_chunks: each chunk's first row in
//                    the columns the mask already compacted
//   select-first     the same, then k_mask_select: the kept rows' pre-mask ids
//
// A kept-row count that the mask contradicts must fail without touching
// memory past what n_valid sizes: the prologue's total is checked (flag 0)
// and so is k_bases' total (flag 1); k_hist and k_scatter read both flags
// first and do nothing when either is set.  The caller sees host_out and
// raises.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "common.cuh"

namespace pf {
namespace {

constexpr int PT = 512;          // threads per CTA
#ifndef PF_PART_ITEMS
#define PF_PART_ITEMS 4
#endif
#ifndef PF_PART_STAGE_RB
#define PF_PART_STAGE_RB 8
#endif
// 2048-row sub-tiles staging at most 8 bytes a row keep the scatter's shared
// memory small enough for several CTAs a SM
constexpr int PITEMS = PF_PART_ITEMS;  // rows per thread per sub-tile
constexpr int SUB = PT * PITEMS; // rows per sub-tile
constexpr int PW = PT / 32;      // warps
constexpr int WSEG = 32 * PITEMS;  // rows of a warp's segment of a sub-tile
constexpr int MAXC = PF_PART_MAX_COLS;
constexpr int MAXCLS = PF_PART_MAX_WIDTHS;
constexpr int BMAX = PF_PART_B_MAX;
constexpr int STAGE_MAX_RB = PF_PART_STAGE_RB;  // rows up to this width are staged in smem

struct Cols {
  const unsigned char* in[MAXC];
  unsigned char* out[MAXC];
  int rb[MAXC];    // bytes a row
  int word[MAXC];  // bytes a copy moves at once (divides rb and both pointers)
  int comp[MAXC];  // 1: n_valid rows, already compacted by the mask
  int cls[MAXC];   // row-width class
  int ncols;
};

struct Params {
  Cols c;
  long long* gout;
  int gcls;
  long long goff;
  const long long* key;
  int key_comp;
  const unsigned char* mask;  // null: every domain row is kept
  long long ndom;             // rows of the walked domain
  const int* src;             // select-first: pre-mask row of kept row j
  long long chunk;            // rows a CTA walks (a multiple of SUB)
  int nchunks;
  const long long* coff;      // compacted-input: each chunk's first compact row
  int needs_j;                // some compacted column is read through coff
  int B, logB, ncls;
  int* hist;                  // [nchunks][B]; exclusive offsets after k_scan
  const long long* bases;     // [MAXCLS][B] padded start of each bucket
  const int* flags;           // [0] prologue count mismatch, [1] overflow
  int stage_rb;               // widest staged row (0: none)
};

// Per sub-tile: every row's rank among the kept rows of the sub-tile (rows in
// warp segments, item k of lane l at w*WSEG + k*32 + l), and their total.
// Holds two __syncthreads.
__device__ __forceinline__ int kept_ranks(const bool (&valid)[PITEMS], int (&rank)[PITEMS],
                                          int* wtot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  int run = 0;
#pragma unroll
  for (int k = 0; k < PITEMS; ++k) {
    const unsigned bal = __ballot_sync(FULL, valid[k]);
    rank[k] = run + __popc(bal & lt);
    run += __popc(bal);
  }
  if (lane == 0) wtot[w] = run;
  __syncthreads();
  int pre = 0, tot = 0;
#pragma unroll
  for (int q = 0; q < PW; ++q) {
    const int t = wtot[q];
    pre += q < w ? t : 0;
    tot += t;
  }
#pragma unroll
  for (int k = 0; k < PITEMS; ++k) rank[k] += pre;
  __syncthreads();  // wtot is reused by the next call
  return tot;
}

// The column index of domain row i for a raw or a compacted column.
__device__ __forceinline__ long long raw_index(const Params& p, long long i) {
  return p.src ? (long long)p.src[i] : i;
}
__device__ __forceinline__ long long comp_index(const Params& p, long long i, long long kept_at) {
  return p.src ? i : kept_at;
}

__device__ __forceinline__ bool failed(const Params& p) {
  return p.flags[0] != 0 || p.flags[1] != 0;
}

// ---- prologues ---------------------------------------------------------------

// Kept rows of each chunk of the pre-mask rows.
__global__ void __launch_bounds__(PT) k_mask_count(const unsigned char* __restrict__ mask,
                                                   long long n, long long chunk,
                                                   long long* __restrict__ cnt) {
  const long long lo = (long long)blockIdx.x * chunk;
  const long long hi = min(n, lo + chunk);
  long long c = 0;
  const bool vec = (((uintptr_t)(mask + lo)) & 15) == 0;
  if (vec) {
    const long long nv = (hi - lo) / 16;
    const uint4* m4 = reinterpret_cast<const uint4*>(mask + lo);
    for (long long v = threadIdx.x; v < nv; v += PT) {
      uint4 x = m4[v];
      const unsigned w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        // non-zero bytes of the word
        const unsigned y = w[q];
        c += ((y & 0xffu) != 0) + ((y & 0xff00u) != 0) + ((y & 0xff0000u) != 0) +
             ((y & 0xff000000u) != 0);
      }
    }
    for (long long i = lo + nv * 16 + threadIdx.x; i < hi; i += PT) c += mask[i] != 0;
  } else {
    for (long long i = lo + threadIdx.x; i < hi; i += PT) c += mask[i] != 0;
  }
  __shared__ long long red[PW];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int q = 0; q < PW; ++q) s += red[q];
    cnt[blockIdx.x] = s;
  }
}

// One block: exclusive scan in place over n chunk counts; total into
// *total; flag 0 when it is not `expect`.
__global__ void __launch_bounds__(1024) k_scan_chunks(long long* __restrict__ a, int n,
                                                      long long expect, int* flags,
                                                      long long* total) {
  __shared__ long long wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int per = (n + 1023) / 1024;
  const int st = tid * per;
  long long s = 0;
  for (int q = 0; q < per; ++q) {
    const int i = st + q;
    if (i < n) s += a[i];
  }
  long long incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const long long v = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    long long v = wsum[lane];
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(FULL, x, o);
      if (lane >= o) x += y;
    }
    wsum[lane] = x - v;  // exclusive prefix of the warps
    if (lane == 31) {
      *total = x;
      if (x != expect) flags[0] = 1;
    }
  }
  __syncthreads();
  long long ex = wsum[w] + incl - s;
  for (int q = 0; q < per; ++q) {
    const int i = st + q;
    if (i < n) {
      const long long t = a[i];
      a[i] = ex;
      ex += t;
    }
  }
}

// select-first: src[k] = the pre-mask row of kept row k, for k < cap.
__global__ void __launch_bounds__(PT) k_mask_select(const unsigned char* __restrict__ mask,
                                                    long long n, long long chunk,
                                                    const long long* __restrict__ coff,
                                                    int* __restrict__ src, long long cap) {
  __shared__ int wtot[PW];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long lo = (long long)blockIdx.x * chunk;
  const long long hi = min(n, lo + chunk);
  long long at = coff[blockIdx.x];
  for (long long sb = lo; sb < hi; sb += SUB) {
    bool valid[PITEMS];
    int rank[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const long long i = sb + w * WSEG + k * 32 + lane;
      valid[k] = i < hi && mask[i] != 0;
    }
    const int tot = kept_ranks(valid, rank, wtot);
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      if (valid[k]) {
        const long long o = at + rank[k];
        if (o < cap) src[o] = (int)(sb + w * WSEG + k * 32 + lane);
      }
    }
    at += tot;
  }
}

// ---- K1: chunk histograms ---------------------------------------------------

__global__ void __launch_bounds__(PT) k_hist(Params p) {
  if (failed(p)) return;
  __shared__ int h[BMAX];
  __shared__ int wtot[PW];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int b = tid; b < p.B; b += PT) h[b] = 0;
  __syncthreads();
  const long long lo = (long long)blockIdx.x * p.chunk;
  const long long hi = min(p.ndom, lo + p.chunk);
  long long kept_at = p.needs_j ? p.coff[blockIdx.x] : 0;
  for (long long sb = lo; sb < hi; sb += SUB) {
    bool valid[PITEMS];
    int rank[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const long long i = sb + w * WSEG + k * 32 + lane;
      bool v = i < hi;
      if (v && p.mask) v = p.mask[i] != 0;
      valid[k] = v;
      rank[k] = 0;
    }
    int tot = 0;
    if (p.key_comp && !p.src) tot = kept_ranks(valid, rank, wtot);
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      if (valid[k]) {
        const long long i = sb + w * WSEG + k * 32 + lane;
        const long long ix = p.key_comp ? comp_index(p, i, kept_at + rank[k]) : raw_index(p, i);
        const int b = bucket_of_hash(mix64((uint64_t)p.key[ix]), p.logB);
        atomicAdd(&h[b], 1);
      }
    }
    kept_at += tot;
  }
  __syncthreads();
  int* row = p.hist + (long long)blockIdx.x * p.B;
  for (int b = tid; b < p.B; b += PT) row[b] = h[b];
}

// The histogram of the plain case (no mask, one sub-tile a chunk): every
// thread's keys loaded first, then counted.
__global__ void __launch_bounds__(PT) k_hist_plain(Params p) {
  if (failed(p)) return;
  __shared__ int h[BMAX];
  const int tid = threadIdx.x;
  for (int b = tid; b < p.B; b += PT) h[b] = 0;
  const long long t0 = (long long)blockIdx.x * SUB;
  long long kv[PITEMS];
#pragma unroll
  for (int k = 0; k < PITEMS; ++k) {
    const long long i = t0 + k * PT + tid;
    kv[k] = i < p.ndom ? p.key[i] : 0;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PITEMS; ++k)
    if (t0 + k * PT + tid < p.ndom) atomicAdd(&h[bucket_of_hash(mix64((uint64_t)kv[k]), p.logB)], 1);
  __syncthreads();
  int* row = p.hist + (long long)blockIdx.x * p.B;
  for (int b = tid; b < p.B; b += PT) row[b] = h[b];
}

// ---- K2: per-bucket offsets over the chunks ---------------------------------

// The chunks are cut into SCAN_G groups; block (x, y) owns buckets
// [32x, 32x + 32) (lane = bucket) of group y, its warps splitting the group's
// chunks.  k_scan_sum: each group's rows a bucket; k_scan_groups: per bucket,
// each group's first row (exclusive over the groups) and counts[b], the
// bucket's rows; k_scan_write: every chunk's exclusive offset into hist.
constexpr int SCAN_G = 64;

__device__ __forceinline__ void scan_range(int nchunks, int cg, int& c0, int& c1) {
  const int g0 = blockIdx.y * cg, g1 = min(nchunks, g0 + cg);
  const int per = (max(0, g1 - g0) + PW - 1) / PW;
  c0 = min(g1, g0 + (threadIdx.x >> 5) * per);
  c1 = min(g1, c0 + per);
}

__global__ void __launch_bounds__(PT) k_scan_sum(const int* __restrict__ hist, int nchunks, int B,
                                                 int cg, long long* __restrict__ gsum,
                                                 const int* flags) {
  if (flags[0]) return;
  __shared__ long long part[PW][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * 32 + lane;
  int c0, c1;
  scan_range(nchunks, cg, c0, c1);
  long long s = 0;
  if (b < B)
    for (int c = c0; c < c1; ++c) s += hist[(long long)c * B + b];
  part[w][lane] = s;
  __syncthreads();
  if (w == 0 && b < B) {
    long long t = 0;
    for (int j = 0; j < PW; ++j) t += part[j][lane];
    gsum[(long long)blockIdx.y * B + b] = t;
  }
}

__global__ void k_scan_groups(long long* __restrict__ gsum, int B, long long* __restrict__ counts,
                              const int* flags) {
  if (flags[0]) return;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  long long run = 0;
  for (int g = 0; g < SCAN_G; ++g) {
    const long long t = gsum[(long long)g * B + b];
    gsum[(long long)g * B + b] = run;
    run += t;
  }
  counts[b] = run;
}

__global__ void __launch_bounds__(PT) k_scan_write(int* __restrict__ hist, int nchunks, int B,
                                                   int cg, const long long* __restrict__ gsum,
                                                   const int* flags) {
  if (flags[0]) return;
  __shared__ long long part[PW][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * 32 + lane;
  const bool live = b < B;
  int c0, c1;
  scan_range(nchunks, cg, c0, c1);
  long long s = 0;
  if (live)
    for (int c = c0; c < c1; ++c) s += hist[(long long)c * B + b];
  part[w][lane] = s;
  __syncthreads();
  if (w == 0) {
    long long run = live ? gsum[(long long)blockIdx.y * B + b] : 0;
    for (int j = 0; j < PW; ++j) {
      const long long t = part[j][lane];
      part[j][lane] = run;
      run += t;
    }
  }
  __syncthreads();
  if (live) {
    long long run = part[w][lane];
    for (int c = c0; c < c1; ++c) {
      const long long i = (long long)c * B + b;
      const int t = hist[i];
      hist[i] = (int)run;
      run += t;
    }
  }
}

// ---- K2b: padded bases, host counts -------------------------------------------

struct Rpu {
  long long v[MAXCLS];
};

// One block of 1024.  host[b] = count b; host[B + cls] = the class's padded
// total; host[B + MAXCLS] = the prologue's kept rows or -1.  Flag 1 when the
// counts total more than n_valid.
__global__ void __launch_bounds__(1024) k_bases(const long long* __restrict__ counts, int B,
                                                Rpu rpu, int ncls, long long* __restrict__ bases,
                                                long long* host, int* flags, long long n_valid,
                                                const long long* prologue_total) {
  __shared__ long long wsum[32];
  __shared__ long long grand;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int per = (B + 1023) / 1024;
  const int st = tid * per;
  const bool bad = flags[0] != 0;
  for (int cls = -1; cls < ncls; ++cls) {
    // cls -1: the raw counts (their total); else the class's padded sizes
    const long long r = cls < 0 ? 1 : rpu.v[cls];
    long long s = 0;
    for (int q = 0; q < per; ++q) {
      const int b = st + q;
      if (b < B) {
        const long long n = bad ? 0 : counts[b];
        s += n ? (n + r - 1) / r * r : 0;
      }
    }
    long long incl = s;
    for (int o = 1; o < 32; o <<= 1) {
      const long long v = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      const long long v = wsum[lane];
      long long x = v;
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
      }
      wsum[lane] = x - v;
      if (lane == 31) grand = x;
    }
    __syncthreads();
    long long ex = wsum[w] + incl - s;
    for (int q = 0; q < per; ++q) {
      const int b = st + q;
      if (b < B) {
        const long long n = bad ? 0 : counts[b];
        if (cls < 0) {
          host[b] = n;
        } else {
          bases[(long long)cls * B + b] = ex;
          ex += n ? (n + r - 1) / r * r : 0;
        }
      }
    }
    if (tid == 0) {
      if (cls < 0) {
        if (grand > n_valid) flags[1] = 1;
        host[B + MAXCLS] = prologue_total ? *prologue_total : -1;
      } else {
        host[B + cls] = grand;
      }
    }
    __syncthreads();
  }
}

// ---- K3: the scatter ---------------------------------------------------------

template <typename T>
__device__ __forceinline__ void stage_rows(const Params& p, int c, const bool (&valid)[PITEMS],
                                           const int (&slot)[PITEMS], const int (&rank)[PITEMS],
                                           long long sb, long long kept_at, T* stage, int nw) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const T* in = reinterpret_cast<const T*>(p.c.in[c]);
  const bool comp = p.c.comp[c] != 0;
  if (nw == 1) {
    // one word a row: every row's load issued before any is stored
    T v[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      if (valid[k]) {
        const long long i = sb + w * WSEG + k * 32 + lane;
        v[k] = in[comp ? comp_index(p, i, kept_at + rank[k]) : raw_index(p, i)];
      }
    }
#pragma unroll
    for (int k = 0; k < PITEMS; ++k)
      if (valid[k]) stage[slot[k]] = v[k];
    return;
  }
#pragma unroll
  for (int k = 0; k < PITEMS; ++k) {
    if (valid[k]) {
      const long long i = sb + w * WSEG + k * 32 + lane;
      const long long ix = comp ? comp_index(p, i, kept_at + rank[k]) : raw_index(p, i);
      const T* row = in + ix * nw;
      T* dst = stage + (long long)slot[k] * nw;
      for (int q = 0; q < nw; ++q) dst[q] = row[q];
    }
  }
}

template <typename T>
__device__ __forceinline__ void write_runs(const Params& p, int c, const T* stage, int nw,
                                           int tvalid, const unsigned short* sbk,
                                           const long long* gbc) {
  T* out = reinterpret_cast<T*>(p.c.out[c]);
  const int n = tvalid * nw;
  if (nw == 1) {
    // n <= SUB: PITEMS staged rows a thread, their lookups unrolled together
#pragma unroll
    for (int t = 0; t < PITEMS; ++t) {
      const int e = t * PT + threadIdx.x;
      if (e < n) out[gbc[sbk[e]] + e] = stage[e];
    }
  } else {
    for (int e = threadIdx.x; e < n; e += PT) {
      const int s = e / nw, q = e - s * nw;
      out[(gbc[sbk[s]] + s) * nw + q] = stage[e];
    }
  }
}

// Rows wider than STAGE_MAX_RB go straight from their source row to their
// output slot, word by word, consecutive threads on consecutive words.
template <typename T>
__device__ __forceinline__ void copy_wide(const Params& p, int c, int nw, int tvalid, long long sb,
                                          long long kept_at, const unsigned short* sbk,
                                          const unsigned short* srow, const unsigned short* skr,
                                          const long long* gbc) {
  const T* in = reinterpret_cast<const T*>(p.c.in[c]);
  T* out = reinterpret_cast<T*>(p.c.out[c]);
  const bool comp = p.c.comp[c] != 0;
  const long long n = (long long)tvalid * nw;
  for (long long e = threadIdx.x; e < n; e += PT) {
    const int s = (int)(e / nw), q = (int)(e - (long long)s * nw);
    const long long i = sb + srow[s];
    const long long ix = comp ? comp_index(p, i, kept_at + skr[s]) : raw_index(p, i);
    out[(gbc[sbk[s]] + s) * nw + q] = in[ix * nw + q];
  }
}

// Dynamic shared memory of k_scatter at B buckets and a widest staged row of
// stage_rb bytes.
size_t scatter_smem(int B, int stage_rb) {
  size_t s = 0;
  s += (size_t)MAXCLS * B * 8;   // gb
  s += (size_t)B * 8;            // run
  s += (size_t)PW * B * 2;       // wcnt
  s += (size_t)2 * B * 4;        // tcnt, tstart
  s += (size_t)3 * SUB * 2;      // sbk, srow, skr
  s += 64 * 4;                   // wtot, misc
  s = (s + 15) / 16 * 16;
  s += (size_t)SUB * stage_rb;   // stage
  return s;
}

// The scatter for the plain case: no mask, one sub-tile a chunk, every column
// one word a row (1, 2, 4 or 8 bytes).  The same stable ranking and staging
// as k_scatter with less state a thread: a CTA a chunk, its rows' buckets,
// warp ranks, the tile's bucket runs, then each column loaded, staged and
// written out with every thread's rows unrolled.
struct PlainSmem {
  unsigned long long stage[SUB];
  long long gb[MAXCLS][BMAX];
  int wh[PW][BMAX];
  int tcnt[BMAX], tstart[BMAX];
  unsigned short sbk[SUB], srow[SUB];
  int wtot[PW];
  int tvalid;
};

// A column of the plain case moves in three steps: its rows loaded into
// registers (widened to 8 bytes), staged in bucket order, written out. The
// next column's loads are issued before this column's write-out.
__device__ __forceinline__ void plain_load(const Params& p, int c, long long t0,
                                           const bool (&valid)[PITEMS],
                                           unsigned long long (&v)[PITEMS]) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const unsigned char* in = p.c.in[c];
  const long long r0 = t0 + w * WSEG + lane;
  switch (p.c.rb[c]) {
    case 8:
#pragma unroll
      for (int k = 0; k < PITEMS; ++k)
        if (valid[k]) v[k] = reinterpret_cast<const unsigned long long*>(in)[r0 + k * 32];
      break;
    case 4:
#pragma unroll
      for (int k = 0; k < PITEMS; ++k)
        if (valid[k]) v[k] = reinterpret_cast<const unsigned*>(in)[r0 + k * 32];
      break;
    case 2:
#pragma unroll
      for (int k = 0; k < PITEMS; ++k)
        if (valid[k]) v[k] = reinterpret_cast<const unsigned short*>(in)[r0 + k * 32];
      break;
    default:
#pragma unroll
      for (int k = 0; k < PITEMS; ++k)
        if (valid[k]) v[k] = in[r0 + k * 32];
      break;
  }
}

template <typename T>
__device__ __forceinline__ void plain_stage(PlainSmem& S, const int (&slot)[PITEMS],
                                            const bool (&valid)[PITEMS],
                                            const unsigned long long (&v)[PITEMS]) {
  T* stage = reinterpret_cast<T*>(S.stage);
#pragma unroll
  for (int k = 0; k < PITEMS; ++k)
    if (valid[k]) stage[slot[k]] = (T)v[k];
}

// eb[t]: the bucket of staged row t*PT + tid (read once for all columns)
template <typename T>
__device__ __forceinline__ void plain_write(const PlainSmem& S, unsigned char* out_,
                                            const long long* gbc, int tvalid,
                                            const int (&eb)[PITEMS]) {
  const T* stage = reinterpret_cast<const T*>(S.stage);
  T* out = reinterpret_cast<T*>(out_);
#pragma unroll
  for (int t = 0; t < PITEMS; ++t) {
    const int e = t * PT + threadIdx.x;
    if (e < tvalid) out[gbc[eb[t]] + e] = stage[e];
  }
}

#ifndef PF_PART_PLAIN_MINB
#define PF_PART_PLAIN_MINB 2  // two blocks a SM: at most 64 registers a thread
#endif
__global__ void __launch_bounds__(PT, PF_PART_PLAIN_MINB) k_scatter_plain(Params p) {
  if (failed(p)) return;
  extern __shared__ __align__(16) unsigned char plain_smem[];
  PlainSmem& S = *reinterpret_cast<PlainSmem*>(plain_smem);
  const int B = p.B;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const long long t0 = (long long)blockIdx.x * SUB;
  for (int x = tid; x < PW * BMAX; x += PT) (&S.wh[0][0])[x] = 0;
  bool valid[PITEMS];
  int bk[PITEMS];
  unsigned long long v[PITEMS];
  {
    long long kv[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const long long i = t0 + w * WSEG + k * 32 + lane;
      valid[k] = i < p.ndom;
      kv[k] = valid[k] ? p.key[i] : 0;
    }
    // the first column rides with the keys (the key column itself: no reload)
    if ((const void*)p.c.in[0] == (const void*)p.key && p.c.rb[0] == 8) {
#pragma unroll
      for (int k = 0; k < PITEMS; ++k) v[k] = (unsigned long long)kv[k];
    } else {
      plain_load(p, 0, t0, valid, v);
    }
#pragma unroll
    for (int k = 0; k < PITEMS; ++k)
      bk[k] = valid[k] ? bucket_of_hash(mix64((uint64_t)kv[k]), p.logB) : -1;
  }
  __syncthreads();
  // stable rank inside (warp, bucket): lane order within an item, items in order
  int sk[PITEMS];
  {
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const unsigned peers = __match_any_sync(FULL, bk[k]);
      const int before = __popc(peers & lt);
      const int base = bk[k] >= 0 ? S.wh[w][bk[k]] : 0;
      __syncwarp();
      if (bk[k] >= 0 && before == 0) S.wh[w][bk[k]] = base + __popc(peers);
      __syncwarp();
      sk[k] = base + before;
    }
  }
  __syncthreads();
  // each warp's start inside the tile's run of every bucket
  for (int b = tid; b < B; b += PT) {
    int r = 0;
#pragma unroll
    for (int q = 0; q < PW; ++q) {
      const int t = S.wh[q][b];
      S.wh[q][b] = r;
      r += t;
    }
    S.tcnt[b] = r;
  }
  __syncthreads();
  // the tile's bucket runs in bucket order (B <= PT: a bucket a thread)
  {
    const int v = tid < B ? S.tcnt[tid] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) S.wtot[w] = incl;
    __syncthreads();
    int pre = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < PW; ++q) {
      const int t = S.wtot[q];
      pre += q < w ? t : 0;
      tot += t;
    }
    if (tid < B) S.tstart[tid] = pre + incl - v;
    if (tid == 0) S.tvalid = tot;
    __syncthreads();
  }
  const int* hrow = p.hist + (long long)blockIdx.x * B;
  for (int x = tid; x < p.ncls * B; x += PT) {
    const int cl = x / B, b = x - cl * B;
    S.gb[cl][b] = p.bases[(long long)cl * B + b] + hrow[b] - S.tstart[b];
  }
  int slot[PITEMS];
#pragma unroll
  for (int k = 0; k < PITEMS; ++k) {
    slot[k] = 0;
    if (bk[k] >= 0) {
      const int s = S.tstart[bk[k]] + S.wh[w][bk[k]] + sk[k];
      slot[k] = s;
      S.sbk[s] = (unsigned short)bk[k];
      S.srow[s] = (unsigned short)(w * WSEG + k * 32 + lane);
    }
  }
  __syncthreads();
  const int tvalid = S.tvalid;
  int eb[PITEMS];
#pragma unroll
  for (int t = 0; t < PITEMS; ++t) {
    const int e = t * PT + tid;
    eb[t] = e < tvalid ? S.sbk[e] : 0;
  }
  for (int c = 0; c < p.c.ncols; ++c) {
    const long long* gbc = S.gb[p.c.cls[c]];
    const int rb = p.c.rb[c];
    unsigned char* out = p.c.out[c];
    switch (rb) {
      case 8: plain_stage<unsigned long long>(S, slot, valid, v); break;
      case 4: plain_stage<unsigned>(S, slot, valid, v); break;
      case 2: plain_stage<unsigned short>(S, slot, valid, v); break;
      default: plain_stage<unsigned char>(S, slot, valid, v); break;
    }
    __syncthreads();
    if (c + 1 < p.c.ncols) plain_load(p, c + 1, t0, valid, v);
    switch (rb) {
      case 8: plain_write<unsigned long long>(S, out, gbc, tvalid, eb); break;
      case 4: plain_write<unsigned>(S, out, gbc, tvalid, eb); break;
      case 2: plain_write<unsigned short>(S, out, gbc, tvalid, eb); break;
      default: plain_write<unsigned char>(S, out, gbc, tvalid, eb); break;
    }
    __syncthreads();
  }
  const long long* gbg = S.gb[p.gcls];
#pragma unroll
  for (int t = 0; t < PITEMS; ++t) {
    const int e = t * PT + tid;
    if (e < tvalid) p.gout[gbg[eb[t]] + e] = p.goff + t0 + S.srow[e];
  }
}

__global__ void __launch_bounds__(PT) k_scatter(Params p) {
  if (failed(p)) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int B = p.B;
  long long* gb = reinterpret_cast<long long*>(smem);   // [MAXCLS][B]
  long long* run = gb + MAXCLS * B;                      // [B]
  unsigned short* wcnt = reinterpret_cast<unsigned short*>(run + B);  // [PW][B]
  int* tcnt = reinterpret_cast<int*>(wcnt + PW * B);     // [B]
  int* tstart = tcnt + B;                                // [B]
  unsigned short* sbk = reinterpret_cast<unsigned short*>(tstart + B);  // [SUB]
  unsigned short* srow = sbk + SUB;                                     // [SUB]
  unsigned short* skr = srow + SUB;                                     // [SUB]
  int* wtot = reinterpret_cast<int*>(skr + SUB);         // [32]
  int* misc = wtot + 32;                                 // [32]
  size_t off = (size_t)(reinterpret_cast<unsigned char*>(misc + 32) - smem);
  off = (off + 15) / 16 * 16;
  unsigned char* stage = smem + off;

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int x = tid; x < PW * B; x += PT) wcnt[x] = 0;
  const unsigned lt = lanemask_lt();
  // the chunks in turn (chunk ch, ch + grid, ...)
  for (int ch = blockIdx.x; ch < p.nchunks; ch += gridDim.x) {
  const int* hrow = p.hist + (long long)ch * B;
  for (int b = tid; b < B; b += PT) run[b] = hrow[b];
  __syncthreads();

  const long long lo = (long long)ch * p.chunk;
  const long long hi = min(p.ndom, lo + p.chunk);
  long long kept_at = p.needs_j ? p.coff[ch] : 0;

  for (long long sb = lo; sb < hi; sb += SUB) {
    bool valid[PITEMS];
    int rank[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const long long i = sb + w * WSEG + k * 32 + lane;
      bool v = i < hi;
      if (v && p.mask) v = p.mask[i] != 0;
      valid[k] = v;
      rank[k] = 0;
    }
    int ktot = 0;
    if (p.needs_j) ktot = kept_ranks(valid, rank, wtot);
    int bk[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      bk[k] = -1;
      if (valid[k]) {
        const long long i = sb + w * WSEG + k * 32 + lane;
        const long long ix = p.key_comp ? comp_index(p, i, kept_at + rank[k]) : raw_index(p, i);
        bk[k] = bucket_of_hash(mix64((uint64_t)p.key[ix]), p.logB);
      }
    }
    // Stable rank inside (warp, bucket): lanes holding the same bucket in
    // one item, in lane order, after the warp's earlier items.
    int wr[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      const unsigned peers = __match_any_sync(FULL, bk[k]);
      const int before = __popc(peers & lt);
      const int base = bk[k] >= 0 ? (int)wcnt[w * B + bk[k]] : 0;
      __syncwarp();
      if (bk[k] >= 0 && before == 0) wcnt[w * B + bk[k]] = (unsigned short)(base + __popc(peers));
      __syncwarp();
      wr[k] = base + before;
    }
    __syncthreads();
    // each warp's start inside the sub-tile's run of every bucket
    for (int b = tid; b < B; b += PT) {
      int r = 0;
#pragma unroll
      for (int q = 0; q < PW; ++q) {
        const int t = wcnt[q * B + b];
        wcnt[q * B + b] = (unsigned short)r;
        r += t;
      }
      tcnt[b] = r;
    }
    __syncthreads();
    // the sub-tile's bucket runs, in bucket order (B <= PT: one bucket a thread)
    {
      const int v = tid < B ? tcnt[tid] : 0;
      int incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wtot[w] = incl;
      __syncthreads();
      int pre = 0, tot = 0;
#pragma unroll
      for (int q = 0; q < PW; ++q) {
        const int t = wtot[q];
        pre += q < w ? t : 0;
        tot += t;
      }
      if (tid < B) tstart[tid] = pre + incl - v;
      if (tid == 0) misc[0] = tot;
      __syncthreads();
    }
    // slot s of bucket b in the sub-tile lands on row gb[cls][b] + s of a
    // class-cls output
    for (int x = tid; x < p.ncls * B; x += PT) {
      const int cl = x / B, b = x - cl * B;
      gb[x] = p.bases[(long long)cl * B + b] + run[b] - tstart[b];
    }
    int slot[PITEMS];
#pragma unroll
    for (int k = 0; k < PITEMS; ++k) {
      slot[k] = 0;
      if (bk[k] >= 0) {
        const int s = tstart[bk[k]] + (int)wcnt[w * B + bk[k]] + wr[k];
        slot[k] = s;
        sbk[s] = (unsigned short)bk[k];
        srow[s] = (unsigned short)(w * WSEG + k * 32 + lane);
        skr[s] = (unsigned short)rank[k];
      }
    }
    __syncthreads();
    const int tvalid = misc[0];

    for (int c = 0; c < p.c.ncols; ++c) {
      const int rb = p.c.rb[c], ws = p.c.word[c], nw = rb / ws;
      const long long* gbc = gb + p.c.cls[c] * B;
      if (rb <= STAGE_MAX_RB) {
        switch (ws) {
          case 8:
            stage_rows<unsigned long long>(p, c, valid, slot, rank, sb, kept_at,
                                           reinterpret_cast<unsigned long long*>(stage), nw);
            __syncthreads();
            write_runs<unsigned long long>(p, c, reinterpret_cast<unsigned long long*>(stage), nw,
                                           tvalid, sbk, gbc);
            break;
          case 4:
            stage_rows<unsigned int>(p, c, valid, slot, rank, sb, kept_at,
                                     reinterpret_cast<unsigned int*>(stage), nw);
            __syncthreads();
            write_runs<unsigned int>(p, c, reinterpret_cast<unsigned int*>(stage), nw, tvalid,
                                     sbk, gbc);
            break;
          case 2:
            stage_rows<unsigned short>(p, c, valid, slot, rank, sb, kept_at,
                                       reinterpret_cast<unsigned short*>(stage), nw);
            __syncthreads();
            write_runs<unsigned short>(p, c, reinterpret_cast<unsigned short*>(stage), nw, tvalid,
                                       sbk, gbc);
            break;
          default:
            stage_rows<unsigned char>(p, c, valid, slot, rank, sb, kept_at, stage, nw);
            __syncthreads();
            write_runs<unsigned char>(p, c, stage, nw, tvalid, sbk, gbc);
            break;
        }
        __syncthreads();
      } else {
        switch (ws) {
          case 8:
            copy_wide<unsigned long long>(p, c, nw, tvalid, sb, kept_at, sbk, srow, skr, gbc);
            break;
          case 4:
            copy_wide<unsigned int>(p, c, nw, tvalid, sb, kept_at, sbk, srow, skr, gbc);
            break;
          case 2:
            copy_wide<unsigned short>(p, c, nw, tvalid, sb, kept_at, sbk, srow, skr, gbc);
            break;
          default:
            copy_wide<unsigned char>(p, c, nw, tvalid, sb, kept_at, sbk, srow, skr, gbc);
            break;
        }
      }
    }
    {
      const long long* gbg = gb + p.gcls * B;
#pragma unroll
      for (int t = 0; t < PITEMS; ++t) {
        const int s = t * PT + tid;
        if (s < tvalid) p.gout[gbg[sbk[s]] + s] = p.goff + raw_index(p, sb + srow[s]);
      }
    }
    __syncthreads();
    for (int b = tid; b < B; b += PT) run[b] += tcnt[b];
    for (int x = tid; x < PW * B; x += PT) wcnt[x] = 0;
    kept_at += ktot;
    __syncthreads();
  }
  }
}

// The chunking of an n-row domain: one sub-tile a chunk, or as few sub-tiles
// as keep the chunk histograms within 2^24 entries.  The scatter's CTAs walk
// the chunks in turn, so the chunks at work at one time are neighbours and
// write next to each other in every bucket (with a long chunk a CTA, every CTA
// kept its own partly written lines in every bucket and column).
void chunking(long long n, int B, long long* chunk, int* nchunks) {
  const long long subs = std::max<long long>(1, (n + SUB - 1) / SUB);
  const long long per = std::max<long long>(1, (subs * B + (1LL << 24) - 1) >> 24);
  *chunk = per * SUB;
  *nchunks = (int)std::max<long long>(1, (n + *chunk - 1) / *chunk);
}

struct Layout {
  int* flags;            // [4]
  long long* pcnt;       // [pre chunks] prologue counts -> offsets
  long long* ptotal;     // [1]
  int* src;              // [n_valid] select-first
  int* hist;             // [nchunks * B]
  long long* gsum;       // [SCAN_G * B]
  long long* counts;     // [B]
  long long* bases;      // [MAXCLS * B]
};

Layout layout(Arena& a, long long n_dom, long long n_valid, int B, bool has_mask,
              bool select_first) {
  Layout l{};
  l.flags = a.take<int>(4);
  l.ptotal = a.take<long long>(1);
  long long pchunk;
  int pn;
  chunking(n_dom, B, &pchunk, &pn);
  l.pcnt = a.take<long long>(has_mask ? pn : 1);
  l.src = a.take<int>(has_mask && select_first ? std::max<long long>(1, n_valid) : 1);
  long long dom = has_mask && select_first ? n_valid : n_dom;
  long long chunk;
  int nch;
  chunking(dom, B, &chunk, &nch);
  if (pn > nch) nch = pn;
  l.hist = a.take<int>((size_t)nch * B);
  l.gsum = a.take<long long>((size_t)SCAN_G * B);
  l.counts = a.take<long long>(B);
  l.bases = a.take<long long>((size_t)MAXCLS * B);
  return l;
}

int word_of(int rb, const void* a, const void* b) {
  for (int w = 8; w > 1; w >>= 1)
    if (rb % w == 0 && ((uintptr_t)a % w) == 0 && ((uintptr_t)b % w) == 0) return w;
  return 1;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_partition_sort_workspace(int64_t n_dom, int64_t n_valid, int B, int has_mask,
                                              int select_first) {
  if (B < 1) B = 1;
  Arena a(nullptr, 0);
  layout(a, n_dom, n_valid, B, has_mask != 0, select_first != 0);
  return a.used + 256;
}

extern "C" int pf_partition_sort(const void* const* cols_in, void* const* cols_out,
                                 const int* row_bytes, const int* comp, int ncols, int key_idx,
                                 const uint8_t* mask, int64_t n_dom, int64_t n_valid, int64_t goff,
                                 int B, int select_first, int64_t* gidx_out, int64_t* host_out,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ncols < 1 || ncols > MAXC) return fail(PF_EINVAL, "partition_sort: 1-%d columns, got %d", MAXC, ncols);
  if (B < 1 || B > BMAX || (B & (B - 1)))
    return fail(PF_EINVAL, "partition_sort: B must be a power of two in [1, %d], got %d", BMAX, B);
  if (key_idx < 0 || key_idx >= ncols) return fail(PF_EINVAL, "partition_sort: key index out of range");
  if (row_bytes[key_idx] != 8) return fail(PF_EINVAL, "partition_sort: the key must be int64");
  if (n_dom < 0 || n_dom >= (1LL << 31))
    return fail(PF_EINVAL, "partition_sort: a call must hold fewer than 2^31 rows, got %lld",
                (long long)n_dom);
  if (n_valid < 0 || n_valid > n_dom)
    return fail(PF_EINVAL, "partition_sort: n_valid %lld outside [0, %lld]", (long long)n_valid,
                (long long)n_dom);
  if (!host_out || !gidx_out) return fail(PF_EINVAL, "partition_sort: null host_out or gidx_out");
  const bool has_mask = mask != nullptr;

  Params p{};
  int rb_cls[MAXCLS];
  int ncls = 0;
  auto cls_of = [&](int rb) -> int {
    for (int c = 0; c < ncls; ++c)
      if (rb_cls[c] == rb) return c;
    if (ncls >= MAXCLS) return -1;
    rb_cls[ncls] = rb;
    return ncls++;
  };
  bool any_comp = false;
  int stage_rb = 0;
  for (int c = 0; c < ncols; ++c) {
    if (row_bytes[c] < 1) return fail(PF_EINVAL, "partition_sort: column %d has empty rows", c);
    if (comp[c] && !has_mask) return fail(PF_EINVAL, "partition_sort: a compacted column needs the mask");
    const int cl = cls_of(row_bytes[c]);
    if (cl < 0) return fail(PF_EINVAL, "partition_sort: more than %d row widths", MAXCLS);
    // an empty column may come with a null pointer (torch gives one for 0 rows)
    const long long in_rows = comp[c] ? n_valid : n_dom;
    const long long out_rows = n_valid + (long long)B * (pf_rows_per_unit(row_bytes[c]) - 1);
    if ((in_rows > 0 && !cols_in[c]) || (out_rows > 0 && !cols_out[c]))
      return fail(PF_EINVAL, "partition_sort: column %d has a null pointer", c);
    p.c.in[c] = (const unsigned char*)cols_in[c];
    p.c.out[c] = (unsigned char*)cols_out[c];
    p.c.rb[c] = row_bytes[c];
    p.c.word[c] = word_of(row_bytes[c], cols_in[c], cols_out[c]);
    p.c.comp[c] = comp[c] ? 1 : 0;
    p.c.cls[c] = cl;
    any_comp |= comp[c] != 0;
    if (row_bytes[c] <= STAGE_MAX_RB) stage_rb = std::max(stage_rb, row_bytes[c]);
  }
  p.c.ncols = ncols;
  p.gcls = cls_of(8);
  if (p.gcls < 0) return fail(PF_EINVAL, "partition_sort: more than %d row widths with the gidx's 8 B", MAXCLS);
  if (((uintptr_t)p.c.in[key_idx] & 7) != 0)
    return fail(PF_EINVAL, "partition_sort: the key column must be 8-byte aligned");
  p.ncls = ncls;
  p.gout = (long long*)gidx_out;
  p.goff = goff;
  p.key = (const long long*)cols_in[key_idx];
  p.key_comp = comp[key_idx] ? 1 : 0;
  p.B = B;
  p.logB = log2_exact((uint64_t)B);
  p.stage_rb = stage_rb;

  const bool use_sel = has_mask && select_first;
  Arena a(workspace, workspace_bytes);
  Layout l = layout(a, n_dom, n_valid, B, has_mask, use_sel);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "partition_sort: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  PF_CUDA(cudaMemsetAsync(l.flags, 0, 4 * sizeof(int), st));
  p.flags = l.flags;
  host_out[B + MAXCLS] = -1;  // no call of ours is in flight: the last one waited

  p.needs_j = any_comp && !use_sel;
  const bool prologue = use_sel || p.needs_j;
  long long pchunk;
  int pn;
  chunking(n_dom, B, &pchunk, &pn);
  if (prologue && n_dom > 0) {
    {
      PF_KERNEL("k_mask_count", st);
      k_mask_count<<<pn, PT, 0, st>>>(mask, n_dom, pchunk, l.pcnt);
    }
    PF_LAUNCH("k_mask_count");
    {
      PF_KERNEL("k_scan_chunks", st);
      k_scan_chunks<<<1, 1024, 0, st>>>(l.pcnt, pn, n_valid, l.flags, l.ptotal);
    }
    PF_LAUNCH("k_scan_chunks");
    if (use_sel) {
      {
        PF_KERNEL("k_mask_select", st);
        k_mask_select<<<pn, PT, 0, st>>>(mask, n_dom, pchunk, l.pcnt, l.src, n_valid);
      }
      PF_LAUNCH("k_mask_select");
    }
  } else if (prologue) {
    PF_CUDA(cudaMemsetAsync(l.ptotal, 0, sizeof(long long), st));
    if (n_valid != 0) PF_CUDA(cudaMemsetAsync(l.flags, 1, 1, st));
  }
  if (use_sel) {
    p.src = l.src;
    p.mask = nullptr;
    p.ndom = n_valid;
  } else {
    p.src = nullptr;
    p.mask = mask;
    p.ndom = n_dom;
    p.coff = l.pcnt;
  }
  chunking(p.ndom, B, &p.chunk, &p.nchunks);
  p.hist = l.hist;
  p.bases = l.bases;

  // the plain case: no mask, one sub-tile a chunk, one word a row
  bool plain = !p.mask && !p.src && !p.needs_j && p.chunk == SUB && !p.key_comp &&
               getenv("PF_PART_GENERAL") == nullptr;
  for (int c = 0; c < p.c.ncols; ++c)
    plain = plain && !p.c.comp[c] && p.c.word[c] == p.c.rb[c] &&
            (p.c.rb[c] == 1 || p.c.rb[c] == 2 || p.c.rb[c] == 4 || p.c.rb[c] == 8);
  {
    PF_KERNEL("k_hist", st);
    if (plain) k_hist_plain<<<p.nchunks, PT, 0, st>>>(p);
    else k_hist<<<p.nchunks, PT, 0, st>>>(p);
  }
  PF_LAUNCH("k_hist");
  {
    const int cg = (p.nchunks + SCAN_G - 1) / SCAN_G;
    const dim3 grid((B + 31) / 32, SCAN_G);
    PF_KERNEL("k_scan", st);
    k_scan_sum<<<grid, PT, 0, st>>>(l.hist, p.nchunks, B, cg, l.gsum, l.flags);
    k_scan_groups<<<(B + 255) / 256, 256, 0, st>>>(l.gsum, B, l.counts, l.flags);
    k_scan_write<<<grid, PT, 0, st>>>(l.hist, p.nchunks, B, cg, l.gsum, l.flags);
  }
  PF_LAUNCH("k_scan");
  Rpu rpu;
  for (int c = 0; c < MAXCLS; ++c) rpu.v[c] = 1;
  for (int c = 0; c < ncls; ++c) rpu.v[c] = pf_rows_per_unit(rb_cls[c]);
  {
    PF_KERNEL("k_bases", st);
    k_bases<<<1, 1024, 0, st>>>(l.counts, B, rpu, ncls, l.bases, host_dev, l.flags, n_valid,
                                prologue ? l.ptotal : nullptr);
  }
  PF_LAUNCH("k_bases");
  cudaEvent_t ev;
  if (int rc = record_event(st, &ev)) return rc;

  if (plain) {
    const size_t smem = sizeof(PlainSmem);
    if (int rc = opt_in_smem((const void*)k_scatter_plain, smem)) return rc;
    {
      PF_KERNEL("k_scatter", st);
      k_scatter_plain<<<p.nchunks, PT, smem, st>>>(p);
    }
    PF_LAUNCH("k_scatter");
    // the call's one host wait: the counts, while the scatter runs
    if (int rc = wait_event(ev)) return rc;
    return ok();
  }
  const size_t smem = scatter_smem(B, stage_rb);
  if (int rc = opt_in_smem((const void*)k_scatter, smem)) return rc;
  {
    // one CTA a chunk: the block scheduler starts the next chunk's loads on a
    // SM while the CTA there still writes out its own
    PF_KERNEL("k_scatter", st);
    k_scatter<<<p.nchunks, PT, smem, st>>>(p);
  }
  PF_LAUNCH("k_scatter");
  // the call's one host wait: the counts, while the scatter runs
  if (int rc = wait_event(ev)) return rc;
  return ok();
}
