// The fused join -> group-by of one unique-build FK join, sm_100a:
//
//   SELECT b.group, SUM(p.price * (scale - p.disc)), COUNT(*)
//   FROM build b JOIN probe p ON b.key = p.fk GROUP BY b.group
//
// It replaces the reference's composition of partition_sort per morsel ->
// join_unique_hash per bucket pair -> index_select -> KeyedAggregate.pass1 ->
// reduce_tick_slice (uvm/join.py:98-225, uvm/aggregate.py:147-212), whose
// every step is an HBM round trip, with these passes:
//
//   1. k_fhist      per-chunk bucket histograms of both sides' keys
//   2. k_fscan      per bucket, each chunk's offset (then the bucket starts)
//   3. k_fscatter   radix scatter of both sides into bucket order; the probe
//                   side carries (fk, value) with value = price * (scale -
//                   disc) computed on the way, so the price and discount
//                   columns are read once and never written
//   then one of two joins (PF_JOIN_PATH):
//   4s. smem (the default): the keys leave pass 3 as their mix64 hashes; a
//                   second radix pass (k_p2_hist, k_p2_colsum, k_p2_scatter)
//                   splits every partition into sub-partitions of about 1.4K
//                   build rows, and k_sjoin joins each in a shared-memory
//                   table, adding every matched probe row's value and 1 into
//                   its build row's cell and flushing each build row once
//                   into the dense group slab (sum, count)
//   4r. rounds:     per round, the round's build rows go into an
//                   open-addressing table in L2 (16-byte slots {key, group |
//                   round tag}); each probe row of the round's partitions
//                   looks its key up and adds its value and 1 into the slab
//                   with fire-and-forget atomics.  One launch probes round r
//                   while it builds round r + 1 into the other half of a
//                   double-buffered table
//
// A row's bucket is the top log2(B) bits of mix64(key), as in the reference's
// partition kernel.  A round is a run of whole partitions whose build rows fit
// the table budget (each partition owns a region of twice its build rows,
// load <= 0.5), or one slice of a partition too large for it (its probe rows
// then meet every slice; a unique build key lives in exactly one).  Slots carry
// the round's tag, so the table is cleared once per call, not per round.
// The bucket counts come to the host once, to plan the rounds or the
// sub-partitions.
#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "scan.cuh"
#include "tma.cuh"

namespace pf {
namespace {

constexpr int FT = 512;            // threads of the histogram and scatter
constexpr int FITEMS = 8;
constexpr int FSUB = FT * FITEMS;  // rows of a scatter sub-tile
constexpr int FB_MAX = 4096;       // fan-out limit
constexpr int PT2 = 256;           // threads of build / probe
// Tunables of the round kernel (minimum resident blocks per SM, which caps
// its registers, and the grid in blocks per SM).  One row a thread at a time
// with full occupancy measured fastest on B200: per-thread batches of rows
// lost more to divergent probe chains than they gained in parallelism.
#ifndef PF_PROBE_MINB
#define PF_PROBE_MINB 8
#endif
#ifndef PF_PROBE_GRID
#define PF_PROBE_GRID 8
#endif

// Build rows a round's table half holds (1.2M: two whole partitions of the
// 150M-row build at B = 256, whose scatter is far cheaper than B = 512's).
constexpr long long ROUND_ROWS_DEFAULT = 1200 * 1024;
// 1: the shared-memory join path by default (PF_JOIN_PATH=rounds|smem
// chooses at run time)
#ifndef PF_JOIN_PATH_DEFAULT
#define PF_JOIN_PATH_DEFAULT 1
#endif
// 1: the shared-memory join's table has fingerprinted 4-byte slots
// (PF_SJ_FP=0|1 chooses at run time)
#ifndef PF_SJ_FP_DEFAULT
#define PF_SJ_FP_DEFAULT 0
#endif

struct Slot {
  unsigned long long key;
  unsigned long long tagged;  // (tag << 32) | group offset
};


// ---- 1. histograms ------------------------------------------------------------

__global__ void __launch_bounds__(FT) k_fhist(const long long* __restrict__ key, long long n,
                                              long long chunk, int logB, int B,
                                              int* __restrict__ hist) {
  extern __shared__ int h[];
  for (int b = threadIdx.x; b < B; b += FT) h[b] = 0;
  __syncthreads();
  const long long lo = (long long)blockIdx.x * chunk;
  const long long hi = min(n, lo + chunk);
  for (long long i = lo + threadIdx.x; i < hi; i += FT) {
    const int b = bucket_of_hash(mix64((uint64_t)key[i]), logB);
    atomicAdd(&h[b], 1);
  }
  __syncthreads();
  int* row = hist + (long long)blockIdx.x * B;
  for (int b = threadIdx.x; b < B; b += FT) row[b] = h[b];
}

// ---- 2. per-bucket chunk offsets ------------------------------------------------

// Block g owns buckets [32g, 32g + 32); warp j scans chunks [j*per, ...).
// hist becomes each chunk's offset inside its bucket; counts[b] the bucket's
// rows.
__global__ void __launch_bounds__(FT) k_fscan(int* __restrict__ hist, int nchunks, int B,
                                              long long* __restrict__ counts) {
  constexpr int W = FT / 32;
  __shared__ long long part[W][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * 32 + lane;
  const bool live = b < B;
  const int per = (nchunks + W - 1) / W;
  const int c0 = w * per, c1 = min(nchunks, c0 + per);
  long long s = 0;
  if (live)
    for (int c = c0; c < c1; ++c) s += hist[(long long)c * B + b];
  part[w][lane] = s;
  __syncthreads();
  if (w == 0) {
    long long run = 0;
    for (int j = 0; j < W; ++j) {
      const long long t = part[j][lane];
      part[j][lane] = run;
      run += t;
    }
    if (live) counts[b] = run;
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

// ---- 3. the scatter ---------------------------------------------------------------

// VAL: the carried value's type (int for the build side's group, long long for
// the probe side's computed value).  HASHED: each row carries mix64(key) in
// place of its key (mix64 is a bijection, so equal keys are equal hashes; the
// shared-memory join path reads buckets and slots from it directly).
template <bool PROBE, bool HASHED>
__global__ void __launch_bounds__(FT) k_fscatter(const long long* __restrict__ key,
                                                 const void* __restrict__ v0,
                                                 const long long* __restrict__ v1,
                                                 long long scale, long long n, long long chunk,
                                                 int logB, int B, const int* __restrict__ hist,
                                                 const long long* __restrict__ start,
                                                 long long* __restrict__ okey,
                                                 void* __restrict__ oval) {
  using V = typename std::conditional<PROBE, long long, int>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  long long* base = reinterpret_cast<long long*>(smem);           // [B]
  int* cnt = reinterpret_cast<int*>(base + B);                     // [B]
  int* tstart = cnt + B;                                           // [B]
  int* wsum = tstart + B;                                          // [32]
  unsigned long long* skey = reinterpret_cast<unsigned long long*>(
      smem + ((size_t)B * 16 + 32 * 4 + 15) / 16 * 16);            // [FSUB]
  V* sval = reinterpret_cast<V*>(skey + FSUB);                     // [FSUB]
  unsigned short* sbk = reinterpret_cast<unsigned short*>(sval + FSUB);  // [FSUB]

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int* hrow = hist + (long long)blockIdx.x * B;
  for (int b = tid; b < B; b += FT) base[b] = start[b] + hrow[b];
  const long long lo = (long long)blockIdx.x * chunk;
  const long long hi = min(n, lo + chunk);
  const V* in0 = reinterpret_cast<const V*>(v0);
  V* out0 = reinterpret_cast<V*>(oval);

  for (long long sb = lo; sb < hi; sb += FSUB) {
    for (int b = tid; b < B; b += FT) cnt[b] = 0;
    __syncthreads();
    long long kv[FITEMS];
    V vv[FITEMS];
    int bk[FITEMS], rk[FITEMS];
#pragma unroll
    for (int k = 0; k < FITEMS; ++k) {
      const long long i = sb + k * FT + tid;
      bk[k] = -1;
      if (i < hi) {
        kv[k] = key[i];
        if (PROBE) {
          const long long price = reinterpret_cast<const long long*>(v0)[i];
          vv[k] = (V)(v1 ? (long long)((unsigned long long)price *
                                       (unsigned long long)(scale - v1[i]))
                         : price);
        } else {
          vv[k] = in0[i];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < FITEMS; ++k) {
      const long long i = sb + k * FT + tid;
      if (i < hi) {
        const uint64_t h = mix64((uint64_t)kv[k]);
        if (HASHED) kv[k] = (long long)h;
        bk[k] = bucket_of_hash(h, logB);
        rk[k] = atomicAdd(&cnt[bk[k]], 1);
      }
    }
    __syncthreads();
    // exclusive scan of cnt into tstart (each thread a run of buckets)
    {
      const int per = (B + FT - 1) / FT;
      const int b0 = tid * per;
      int s = 0;
      for (int q = 0; q < per; ++q)
        if (b0 + q < B) s += cnt[b0 + q];
      int incl = s;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[w] = incl;
      __syncthreads();
      int pre = 0;
      for (int q = 0; q < FT / 32; ++q) pre += q < w ? wsum[q] : 0;
      int ex = pre + incl - s;
      for (int q = 0; q < per; ++q) {
        if (b0 + q < B) {
          tstart[b0 + q] = ex;
          ex += cnt[b0 + q];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < FITEMS; ++k) {
      if (bk[k] >= 0) {
        const int s = tstart[bk[k]] + rk[k];
        skey[s] = (unsigned long long)kv[k];
        sval[s] = vv[k];
        sbk[s] = (unsigned short)bk[k];
      }
    }
    __syncthreads();
    const int nsub = (int)min((long long)FSUB, hi - sb);
    for (int s = tid; s < nsub; s += FT) {
      const int b = sbk[s];
      const long long pos = base[b] + (s - tstart[b]);
      okey[pos] = (long long)skey[s];
      out0[pos] = sval[s];
    }
    __syncthreads();
    for (int b = tid; b < B; b += FT) base[b] += cnt[b];
    __syncthreads();
  }
}

size_t fscatter_smem(int B, bool probe) {
  size_t s = ((size_t)B * 16 + 32 * 4 + 15) / 16 * 16;
  s += (size_t)FSUB * 8;                // skey
  s += (size_t)FSUB * (probe ? 8 : 4);  // sval
  s += (size_t)FSUB * 2;                // sbk
  return s;
}

// ---- 3'. the scatter fed by bulk asynchronous copies -----------------------------------

// The same scatter with each 2048-row sub-tile's source columns brought into
// shared memory by bulk copies (the TMA engine) up to TNBUF sub-tiles ahead,
// so the reads of later sub-tiles overlap the ranking, staging and writes of
// the current one.  Used when every source column is 16-byte aligned; the
// bytes of a final partial sub-tile past its last whole 16 come from global
// loads.  A bulk copy that never lands (bounded waits) sets *err and the
// CTA stops after waiting, again bounded, for its copies still in flight.
#ifndef PF_TT
#define PF_TT 512
#endif
#ifndef PF_TSUB_P
#define PF_TSUB_P 2048
#endif
#ifndef PF_TSUB_B
#define PF_TSUB_B 4096
#endif
constexpr int TT = PF_TT;
// rows of a sub-tile: the probe side carries 24 B a row in, the build side 12
template <bool PROBE>
struct TSub {
  static constexpr int rows = PROBE ? PF_TSUB_P : PF_TSUB_B;
};

struct TmaCols {
  const void* src[3];
  int es[3];
  int ncols;
};

template <bool PROBE>
struct TmaSmem {
  static constexpr int TSUB = TSub<PROBE>::rows;
  // offsets (bytes) of each region for B buckets and nbuf buffers
  size_t bar, in, stage_key, stage_val, sbk, base, cnt, tstart, wsum, flag, total;
  size_t in_stride;  // bytes of one buffer
  __host__ __device__ TmaSmem(int B, int nbuf) {
    const size_t rowb = PROBE ? 24 : 12;
    size_t o = 0;
    bar = o;
    o += 128;
    in = o;
    in_stride = (size_t)TSUB * rowb;
    o += (size_t)nbuf * in_stride;
    stage_key = o;
    o += (size_t)TSUB * 8;
    stage_val = o;
    o += (size_t)TSUB * (PROBE ? 8 : 4);
    sbk = o;
    o += (size_t)TSUB * 2;
    o = (o + 15) / 16 * 16;
    base = o;
    o += (size_t)B * 8;
    cnt = o;
    o += (size_t)B * 4;
    tstart = o;
    o += (size_t)B * 4;
    wsum = o;
    o += 32 * 4;
    flag = o;
    o += 16;
    total = (o + 127) / 128 * 128;
  }
};

template <bool PROBE, bool HASHED>
__global__ void __launch_bounds__(TT) k_fscatter_tma(const long long* __restrict__ key,
                                                     const void* __restrict__ v0,
                                                     const long long* __restrict__ v1,
                                                     long long scale, long long n, long long chunk,
                                                     int logB, int B, int nbuf,
                                                     const int* __restrict__ hist,
                                                     const long long* __restrict__ start,
                                                     long long* __restrict__ okey,
                                                     void* __restrict__ oval,
                                                     unsigned long long* err) {
  using V = typename std::conditional<PROBE, long long, int>::type;
  constexpr int TSUB = TSub<PROBE>::rows;
  constexpr int TROWS = TSUB / TT;
  extern __shared__ __align__(128) unsigned char tsmem[];
  const TmaSmem<PROBE> L(B, nbuf);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsmem + L.bar);
  unsigned long long* skey = reinterpret_cast<unsigned long long*>(tsmem + L.stage_key);
  V* sval = reinterpret_cast<V*>(tsmem + L.stage_val);
  unsigned short* sbk = reinterpret_cast<unsigned short*>(tsmem + L.sbk);
  long long* base = reinterpret_cast<long long*>(tsmem + L.base);
  int* cnt = reinterpret_cast<int*>(tsmem + L.cnt);
  int* tstart = reinterpret_cast<int*>(tsmem + L.tstart);
  int* wsum = reinterpret_cast<int*>(tsmem + L.wsum);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const long long lo = (long long)blockIdx.x * chunk;
  const long long hi = min(n, lo + chunk);
  const int ntiles = lo < hi ? (int)((hi - lo + TSUB - 1) / TSUB) : 0;
  const int ncols = PROBE ? (v1 ? 3 : 2) : 2;
  const void* src[3] = {key, v0, v1};
  const int es[3] = {8, PROBE ? 8 : 4, 8};
  // column c of buffer b: in + b*in_stride + colofs[c]
  const size_t colofs[3] = {0, (size_t)TSUB * 8, (size_t)TSUB * (PROBE ? 16 : 12)};

  auto tma_rows = [&](int c, int rows) -> int { return (rows * es[c]) / 16 * 16 / es[c]; };
  auto issue = [&](int t) {
    const int b = t % nbuf;
    const long long sb = lo + (long long)t * TSUB;
    const int rows = (int)min((long long)TSUB, hi - sb);
    unsigned bytes = 0;
    for (int c = 0; c < ncols; ++c) bytes += (unsigned)(tma_rows(c, rows) * es[c]);
    mbar_arrive_expect_tx(&bar[b], bytes);
    for (int c = 0; c < ncols; ++c) {
      const unsigned nb = (unsigned)(tma_rows(c, rows) * es[c]);
      if (nb)
        bulk_g2s(tsmem + L.in + b * L.in_stride + colofs[c],
                 reinterpret_cast<const char*>(src[c]) + sb * es[c], nb, &bar[b]);
    }
  };

  if (tid == 0) {
    for (int b = 0; b < nbuf; ++b) mbar_init(&bar[b], 1);
    mbar_init_fence();
  }
  const int* hrow = hist + (long long)blockIdx.x * B;
  for (int b = tid; b < B; b += TT) base[b] = start[b] + hrow[b];
  __syncthreads();
  if (tid == 0)
    for (int t = 0; t < min(nbuf, ntiles); ++t) issue(t);

  const V* g0 = reinterpret_cast<const V*>(v0);
  V* out0 = reinterpret_cast<V*>(oval);
  for (int t = 0; t < ntiles; ++t) {
    const int b_ = t % nbuf;
    const unsigned parity = (unsigned)((t / nbuf) & 1);
    const long long sb = lo + (long long)t * TSUB;
    const int rows = (int)min((long long)TSUB, hi - sb);
    for (int b = tid; b < B; b += TT) cnt[b] = 0;
    const bool ok = mbar_wait_bounded(&bar[b_], parity);
    if (__syncthreads_or(!ok)) {
      // a copy never landed: report, let the copies in flight finish, stop
      if (tid == 0) {
        atomicOr(err, 1ULL);
        for (int u = t; u < min(ntiles, t + nbuf); ++u)
          mbar_wait_bounded(&bar[u % nbuf], (unsigned)((u / nbuf) & 1), 1u << 16);
      }
      __syncthreads();
      return;
    }
    const unsigned char* ib = tsmem + L.in + b_ * L.in_stride;
    const unsigned long long* ik = reinterpret_cast<const unsigned long long*>(ib + colofs[0]);
    const V* iv = reinterpret_cast<const V*>(ib + colofs[1]);
    const long long* id = reinterpret_cast<const long long*>(ib + colofs[2]);
    const int tk = tma_rows(0, rows), tv = tma_rows(1, rows), td = tma_rows(2, rows);
    unsigned long long kv[TROWS];
    V vv[TROWS];
    int bk[TROWS], rk[TROWS];
#pragma unroll
    for (int k = 0; k < TROWS; ++k) {
      const int r = k * TT + tid;
      bk[k] = -1;
      if (r < rows) {
        kv[k] = r < tk ? ik[r] : (unsigned long long)key[sb + r];
        if (PROBE) {
          const long long price = r < tv ? (long long)iv[r] : reinterpret_cast<const long long*>(v0)[sb + r];
          if (v1) {
            const long long d = r < td ? id[r] : v1[sb + r];
            vv[k] = (V)(long long)((unsigned long long)price * (unsigned long long)(scale - d));
          } else {
            vv[k] = (V)price;
          }
        } else {
          vv[k] = r < tv ? iv[r] : g0[sb + r];
        }
        const uint64_t h = mix64(kv[k]);
        if (HASHED) kv[k] = h;
        bk[k] = bucket_of_hash(h, logB);
        rk[k] = atomicAdd(&cnt[bk[k]], 1);
      }
    }
    __syncthreads();
    {
      const int per = (B + TT - 1) / TT;
      const int b0 = tid * per;
      int s = 0;
      for (int q = 0; q < per; ++q)
        if (b0 + q < B) s += cnt[b0 + q];
      int incl = s;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[w] = incl;
      __syncthreads();
      int pre = 0;
      for (int q = 0; q < TT / 32; ++q) pre += q < w ? wsum[q] : 0;
      int ex = pre + incl - s;
      for (int q = 0; q < per; ++q) {
        if (b0 + q < B) {
          tstart[b0 + q] = ex;
          ex += cnt[b0 + q];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TROWS; ++k) {
      if (bk[k] >= 0) {
        const int s = tstart[bk[k]] + rk[k];
        skey[s] = kv[k];
        sval[s] = vv[k];
        sbk[s] = (unsigned short)bk[k];
      }
    }
    __syncthreads();
    // this buffer is consumed: refill it with the sub-tile nbuf ahead
    if (tid == 0 && t + nbuf < ntiles) {
      fence_proxy_async_smem();
      issue(t + nbuf);
    }
    for (int s = tid; s < rows; s += TT) {
      const int b = sbk[s];
      const long long pos = base[b] + (s - tstart[b]);
      okey[pos] = (long long)skey[s];
      out0[pos] = sval[s];
    }
    __syncthreads();
    for (int b = tid; b < B; b += TT) base[b] += cnt[b];
  }
}

template <bool PROBE>
int tma_nbuf(int B) {
  return TmaSmem<PROBE>(B, 3).total <= 220 * 1024 ? 3 : 2;
}

template <bool PROBE>
size_t tma_smem(int B) {
  return TmaSmem<PROBE>(B, tma_nbuf<PROBE>(B)).total;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// ---- 4. rounds: build and probe ----------------------------------------------------

struct RoundArgs {
  const long long* bkey;  // partitioned build keys
  const int* bgrp;        // partitioned build groups
  long long b_lo, b_hi;   // the round's build rows
  const long long* pfk;   // partitioned probe keys
  const long long* pval;  // partitioned probe values
  long long p_lo, p_hi;   // the round's probe rows
  Slot* table;
  const long long* reg_off;  // [B] slot offset of each partition's region
  const long long* reg_cap;  // [B] slots of each partition's region
  int p0, p1;                // the round's partitions
  long long slice_cap;       // > 0: a slice round, one region of this size at 0
  unsigned tag;
  int logB;
  long long group_min, n_groups;
  unsigned long long* slab;   // [2 * n_groups]: (sum, count) of group g at 2g, 2g+1
  unsigned long long* stats;  // [0] matched, [1] reserved, [2] build rows out of group range, [3] overflow
};

__device__ __forceinline__ uint2 region_of(const RoundArgs& a, const uint2* reg, uint64_t h) {
  return a.slice_cap > 0 ? reg[0] : reg[bucket_of_hash(h, a.logB) - a.p0];
}

// The first slot of hash h inside a region of `cap` slots: multiply-shift of
// the 32 bits right below the bucket bits.
__device__ __forceinline__ unsigned first_slot(uint64_t h, int logB, unsigned cap) {
  const uint32_t x = (uint32_t)((h << logB) >> 32);
  return (unsigned)(((unsigned long long)x * cap) >> 32);
}

__device__ __forceinline__ ulonglong2 ld_slot(const Slot* p) {
  return __ldcg(reinterpret_cast<const ulonglong2*>(p));
}

// 1: the partitioned sides, read once, are loaded evict-first (ld.global.cs)
// so that they do not push the round's tables and the slab out of L2; the
// probe value then travels in a register instead of shared memory.
#ifndef PF_STREAM_HINTS
#define PF_STREAM_HINTS 1
#endif
template <typename T>
__device__ __forceinline__ T stream_ld(const T* p) {
#if PF_STREAM_HINTS
  return __ldcs(p);
#else
  return *p;
#endif
}

// Build one row.  A slot is free for this round when its tag (the high half
// of the tagged word) is below the round's tag (tags grow round by round; the
// table is zeroed once per call): an atomicMax of the tag claims it without a
// read first, and only the claimant, seeing an older tag come back, writes the
// whole slot (key, group, tag) with one 16-byte store.  A loser's max leaves
// the tag as it is.  The round's probe runs in a later launch.
__device__ __forceinline__ void build_row(const RoundArgs& a, const uint2* reg, long long i,
                                          unsigned long long& bad_group,
                                          unsigned long long& overflow) {
  const unsigned long long key = (unsigned long long)stream_ld(a.bkey + i);
  const long long g = (long long)stream_ld(a.bgrp + i) - a.group_min;
  uint32_t goff = 0xffffffffu;
  if (g >= 0 && g < a.n_groups) goff = (uint32_t)g;
  else ++bad_group;
  const uint64_t h = mix64(key);
  const uint2 r = region_of(a, reg, h);
  unsigned pos = first_slot(h, a.logB, r.y);
  for (unsigned left = r.y; left > 0; --left) {
    Slot* sl = a.table + r.x + pos;
    unsigned* tag = reinterpret_cast<unsigned*>(&sl->tagged) + 1;
    if (atomicMax(tag, a.tag) < a.tag) {
      *reinterpret_cast<ulonglong2*>(sl) =
          make_ulonglong2(key, ((unsigned long long)a.tag << 32) | goff);
      return;
    }
    if (++pos == r.y) pos = 0;
  }
  ++overflow;
}

// cp.async (16 or 8 bytes, global -> shared, not through registers).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
#if !PF_STREAM_HINTS
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
#endif
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// Probe PR rows a thread (rows lo + k*PT2 + tid): every row's first slot
// and value are gathered into shared memory by cp.async before any is
// examined, so a thread keeps PR lookups in flight without holding them in
// registers; a collision continues with plain loads.
#ifndef PF_PR
#define PF_PR 2
#endif
constexpr int PR = PF_PR;
constexpr int PUROWS = PT2 * PR;

struct ProbeStage {
  ulonglong2 slot[PR][PT2];
#if !PF_STREAM_HINTS
  long long val[PR][PT2];
#endif
};

__device__ __forceinline__ void probe_unit(const RoundArgs& a, const uint2* reg, long long lo,
                                           long long hi, ProbeStage& st,
                                           unsigned long long& matched) {
  const int tid = threadIdx.x;
  unsigned long long key[PR];
  unsigned pos[PR];
  uint2 rg[PR];
#if PF_STREAM_HINTS
  long long val[PR];
#pragma unroll
  for (int k = 0; k < PR; ++k) {
    const long long i = lo + k * PT2 + tid;
    key[k] = i < hi ? (unsigned long long)stream_ld(a.pfk + i) : 0ULL;
    val[k] = i < hi ? stream_ld(a.pval + i) : 0;
  }
#endif
#pragma unroll
  for (int k = 0; k < PR; ++k) {
    const long long i = lo + k * PT2 + tid;
    rg[k] = make_uint2(0u, 0u);
    if (i < hi) {
#if !PF_STREAM_HINTS
      key[k] = (unsigned long long)a.pfk[i];
#endif
      const uint64_t h = mix64(key[k]);
      rg[k] = region_of(a, reg, h);
      if (rg[k].y) {
        pos[k] = first_slot(h, a.logB, rg[k].y);
        cp_async16(&st.slot[k][tid], a.table + rg[k].x + pos[k]);
#if !PF_STREAM_HINTS
        cp_async8(&st.val[k][tid], a.pval + i);
#endif
      }
    }
  }
  cp_async_wait_all();
#pragma unroll
  for (int k = 0; k < PR; ++k) {
    if (rg[k].y == 0) continue;
    ulonglong2 sl = st.slot[k][tid];
    for (unsigned probes = 1;; ++probes) {
      if ((uint32_t)(sl.y >> 32) != a.tag) break;  // a free slot: no match
      if (sl.x == key[k]) {
        const uint32_t g = (uint32_t)sl.y;
        if (g != 0xffffffffu) {
#if PF_STREAM_HINTS
          atomicAdd(&a.slab[2 * (unsigned long long)g], (unsigned long long)val[k]);
#else
          atomicAdd(&a.slab[2 * (unsigned long long)g], (unsigned long long)st.val[k][tid]);
#endif
          atomicAdd(&a.slab[2 * (unsigned long long)g + 1], 1ULL);
        }
        ++matched;
        break;
      }
      if (probes >= rg[k].y) break;
      if (++pos[k] == rg[k].y) pos[k] = 0;
      sl = ld_slot(a.table + rg[k].x + pos[k]);
    }
  }
}

// One launch of the round pipeline: probe round r (pa, its table half) while
// building round r + 1 (ba, the other half).  Blocks take work units of
// UROWS rows from a per-launch counter; build units are spread evenly among
// the probe units, so the build's claim round trips overlap the probe's L2
// traffic across the whole launch.  Kernel boundaries give the ordering: a
// round's table is complete before its probe launch, and a half is probed to
// the end before the launch that rebuilds it.
constexpr int UROWS = 1024;

__global__ void __launch_bounds__(PT2, PF_PROBE_MINB) k_fround(RoundArgs pa, RoundArgs ba,
                                                             unsigned* counter, int units_p,
                                                             int units_b) {
  extern __shared__ __align__(16) unsigned char fr_smem[];
  __shared__ int unit;
  ProbeStage& stage = *reinterpret_cast<ProbeStage*>(fr_smem);
  uint2* regs = reinterpret_cast<uint2*>(fr_smem + sizeof(ProbeStage));
  const int np = pa.p_hi > pa.p_lo ? (pa.slice_cap > 0 ? 1 : pa.p1 - pa.p0) : 0;
  const int nbr = ba.b_hi > ba.b_lo ? (ba.slice_cap > 0 ? 1 : ba.p1 - ba.p0) : 0;
  uint2* regp = regs;
  uint2* regb = regs + np;
  for (int i = threadIdx.x; i < np; i += blockDim.x)
    regp[i] = pa.slice_cap > 0 ? make_uint2(0u, (unsigned)pa.slice_cap)
                               : make_uint2((unsigned)pa.reg_off[pa.p0 + i],
                                            (unsigned)pa.reg_cap[pa.p0 + i]);
  for (int i = threadIdx.x; i < nbr; i += blockDim.x)
    regb[i] = ba.slice_cap > 0 ? make_uint2(0u, (unsigned)ba.slice_cap)
                               : make_uint2((unsigned)ba.reg_off[ba.p0 + i],
                                            (unsigned)ba.reg_cap[ba.p0 + i]);
  unsigned long long matched = 0, bad_group = 0, overflow = 0;
  const long long U = (long long)units_p + units_b;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) unit = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const long long u = unit;
    if (u >= U) break;
    const long long nb_upto = (u + 1) * units_b / U;  // build units among [0, u]
    const bool build = nb_upto > u * units_b / U;
    if (build) {
      const long long lo = ba.b_lo + (nb_upto - 1) * UROWS;
      const long long hi = min(ba.b_hi, lo + UROWS);
      for (long long i = lo + threadIdx.x; i < hi; i += PT2) build_row(ba, regb, i, bad_group, overflow);
    } else {
      const long long lo = pa.p_lo + (u - nb_upto) * UROWS;
      const long long hi = min(pa.p_hi, lo + UROWS);
      for (long long l0 = lo; l0 < hi; l0 += PUROWS)
        probe_unit(pa, regp, l0, min(hi, l0 + PUROWS), stage, matched);
    }
  }
  for (int o = 16; o; o >>= 1) matched += __shfl_xor_sync(FULL, matched, o);
  if ((threadIdx.x & 31) == 0 && matched) atomicAdd(&pa.stats[0], matched);
  if (bad_group) atomicAdd(&ba.stats[2], bad_group);
  if (overflow) atomicAdd(&ba.stats[3], overflow);
}


// ---- the shared-memory join: a second radix pass, then per sub-partition ----
//
// PF_JOIN_PATH=smem (the default): the first scatter carries each key's mix64
// hash in place of the key (a bijection: equal keys, equal hashes), each
// partition is split again by the next log2(B2) bits of the hash, so every
// sub-partition holds about SJ_TARGET build rows; then k_sjoin takes
// sub-partitions from a counter: it puts the build rows into a shared-memory
// table {hash, sum, count}, adds every matching probe row's value and 1 into
// its build row's cell with shared-memory atomics, and flushes each build row
// that matched into the group slab with one pair of global REDs.  Per probe
// row no L2 operation at all; per build row one pair.  A sub-partition with
// more build rows than the table takes is joined in table-sized chunks of its
// build rows, each chunk against all of its probe rows.  The table marks a
// free slot with the hash INT64_MIN; the key whose hash that is gets a cell of
// its own.
//
// Neither radix pass counts its rows first.  Each (sub-)bucket owns a region
// of the output sized for its expected rows plus seven standard deviations
// (the hash spreads the keys of a side uniformly), and the scatter's cursor
// claims run from the region's start.  A tile whose claim would cross its
// region's end writes none of that bucket's rows and raises the overflow
// word instead; the host sees it and runs that pass again with exact counts
// (per-segment histograms and a scan: the counted passes).  Skewed keys, which
// crowd one bucket, take that route; uniform ones never do.  The probe side
// travels as 16-byte records {hash, value}: one load and one store a row.

// One 1024-thread block a SM with 8192-row tiles: runs of 16 rows at 512
// sub-buckets (measured against 512 threads x 4096 rows: 6.03 vs 6.79 ms for
// the 150M x 600M second pass).
#ifndef PF_P2T
#define PF_P2T 1024
#endif
#ifndef PF_P2I
#define PF_P2I 8
#endif
#ifndef PF_P2_MINB
#define PF_P2_MINB 1
#endif
// Staged rows a thread writes out at a time: two for the build side's
// columns (measured 0.99 -> 0.95 ms for 150M rows), one for the probe side's
// records (two spill there: 5.68 -> 5.96 ms for the second pass)
// > 0: each tile's thread 0 prefetches into L2 (one TMA bulk prefetch a
// column) the rows of the tile that many turns ahead, in the passes that have
// the registers for it (not the build side's second pass, which would spill).
// Measured on 150M x 600M rows: one turn ahead (the tile whose register loads
// this one issues before its write-out) takes the first pass's probe side
// from 4.37 to 4.19 ms and the second pass from 5.09 to 4.98; two turns ahead
// is slower than none (4.71, 5.16), three slower still.
#ifndef PF_P2_L2PF
#define PF_P2_L2PF 1
#endif
// Staged rows a thread writes out at a time in the build side's passes
// (columns, thread stores): two measured 0.99 -> 0.95 ms for the first pass
// over 150M rows
#ifndef PF_P2_WU
#define PF_P2_WU 2
#endif
constexpr int P2T = PF_P2T;
constexpr int P2I = PF_P2I;
constexpr int P2TILE = P2T * P2I;  // rows a tile (the build side's passes)
// The probe side's second pass: rows a thread (its records leave shared
// memory by bulk copies, so no thread holds rows through a write-out; on
// 600M probe rows 9 rows a thread measured 0.08 ms less than 8; 10 and 11
// spill and take 0.33 and 0.56 ms more)
#ifndef PF_P2I_AOS
#define PF_P2I_AOS 9
#endif
constexpr int P2I_AOS = PF_P2I_AOS;
// The first pass's probe side carries three input columns a row into its
// registers: 7 rows a thread (7168-row tiles) keep it within 64 registers
// without spilling (on 600M probe rows: 7 rows 4.85 ms, 6 rows 4.93, 8 rows
// spill and take longer).
#ifndef PF_P2_RI2
#define PF_P2_RI2 7
#endif
constexpr int P2RI2 = PF_P2_RI2;
constexpr int P2MAXLOG = 10;       // sub-buckets a partition splits into, log2, at most
constexpr int P2BINS = 1 << P2MAXLOG;
constexpr int P1BINS = FB_MAX;     // the first pass's buckets, at most
static_assert(P2BINS % P2T == 0 && P1BINS % P2T == 0, "whole bins a thread in the tile scan");
// Three 512-thread blocks a SM, each with a 3072-slot table (63 KB of shared
// memory: hash, two-word sum, count; no group offsets).  Measured on the
// 150M x 600M join: three 384-thread blocks 4.59 ms, three 512-thread blocks
// 4.38 (the kernel waits on shared-memory latency: more warps hide more of
// it), two 512-thread blocks with 4096-slot tables and stored offsets 5.43,
// two 384-thread blocks 7.19, four 384-thread blocks with 2560-slot tables
// 4.58, two 1024-thread blocks 5.17; 3328- or 3584-slot tables (still three
// blocks a SM) within 0.04 ms of 3072.
#ifndef PF_SJT
#define PF_SJT 512
#endif
#ifndef PF_SJ_MINB
#define PF_SJ_MINB 3
#endif
#ifndef PF_SJ_U
#define PF_SJ_U 1
#endif
// 1: the probe loop loads the next round's rows before looking up this one's
#ifndef PF_SJ_PIPE
#define PF_SJ_PIPE 1
#endif
constexpr int SJT = PF_SJT;       // threads of the join
#ifndef PF_SJ_LOGTS
#define PF_SJ_LOGTS 12
#endif
#ifndef PF_SJ_TS
#define PF_SJ_TS 3072
#endif
constexpr int SJ_TS = PF_SJ_TS;                // table slots
constexpr bool SJ_POW2 = (SJ_TS & (SJ_TS - 1)) == 0;
static_assert(!SJ_POW2 || SJ_TS == (1 << PF_SJ_LOGTS), "a power-of-two table is 2^PF_SJ_LOGTS slots");
#ifndef PF_SJ_CAP
#define PF_SJ_CAP (SJ_TS / 2)
#endif
#ifndef PF_SJ_TARGET
#define PF_SJ_TARGET 1365
#endif
constexpr int SJ_CAP = PF_SJ_CAP;              // build rows a table takes
constexpr long long SJ_TARGET = PF_SJ_TARGET;  // build rows a sub-partition aims at
constexpr long long SJ_EMPTY = LLONG_MIN;
constexpr unsigned SJ_NONE = 0xffffffffu;
constexpr int SJ_U = PF_SJ_U;                  // probe rows a thread holds at once
constexpr int SJ_BU = SJ_CAP / SJT;            // build rows a thread takes per chunk
static_assert(SJ_CAP % SJT == 0, "whole build rounds");
static_assert(SJ_TS < 0xffff, "slots fit the 16-bit slot index");

// The counted second pass works on segments: runs of at most P2SEG rows
// inside one partition (segment (p, j) is rows [start_p + j * P2SEG,
// min(start_p + (j + 1) * P2SEG, end_p))), so a segment's rows share their
// partition and its 2^logB2 sub-buckets.
constexpr long long P2SEG = 16LL * P2TILE;

// Rows a (sub-)bucket's region holds for `mean` expected rows: seven
// standard deviations over the mean and a few rows more.  A side of distinct
// keys (the build side) lands binomially, its deviation below sqrt(mean);
// the probe side repeats keys (each build key is met m times on average), so
// its bucket counts vary with the build keys' as well: var ~ mean * (1 + m).
// Its regions allow var = 8 * mean, repeats up to about seven a key; skewed
// keys past that overflow, and the pass is counted instead.
constexpr double REGION_VAR_BUILD = 1.0;
constexpr double REGION_VAR_PROBE = 8.0;
inline long long region_rows(double mean, double var_factor) {
  return (long long)std::ceil(mean + 7.0 * std::sqrt(var_factor * mean)) + 32;
}
inline double region_var(int side) { return side ? REGION_VAR_PROBE : REGION_VAR_BUILD; }

struct SegArgs {
  const int2* seg;          // (partition, index in the partition)
  int nseg;
  const long long* pstart;  // the side's partition starts
  const long long* pcnt;    // and rows
  int logS, logB2;
};

__device__ __forceinline__ void seg_range(const SegArgs& g, int sg, long long& lo, long long& hi,
                                          long long& base) {
  const int2 d = g.seg[sg];
  const long long p0 = g.pstart[d.x];
  lo = p0 + (long long)d.y * P2SEG;
  hi = min(lo + P2SEG, p0 + g.pcnt[d.x]);
  base = (long long)d.x << g.logB2;
}

// A staged row: key (hash) and value in one 16-byte record; the probe side's
// partitioned rows are stored in HBM in the same form.
struct alignas(16) P2Row {
  long long k;
  long long v;
};

__device__ __forceinline__ P2Row stream_ld_row(const P2Row* p) {
  const longlong2 r = stream_ld(reinterpret_cast<const longlong2*>(p));
  return P2Row{r.x, r.y};
}

// Each segment's sub-bucket counts, hist[sg][b] (every one of the 2^logB2
// written, zeros too).  AOS: the side's rows are records.
template <bool AOS>
__global__ void __launch_bounds__(P2T) k_p2_hist(const long long* __restrict__ key,
                                                 const P2Row* __restrict__ rec, SegArgs g,
                                                 int* __restrict__ hist) {
  __shared__ int bins[P2BINS];
  const int nb2 = 1 << g.logB2;
  const int tid = threadIdx.x;
  for (int sg = blockIdx.x; sg < g.nseg; sg += gridDim.x) {
    long long lo, hi, base;
    seg_range(g, sg, lo, hi, base);
    for (int b = tid; b < nb2; b += P2T) bins[b] = 0;
    __syncthreads();
    for (long long t0 = lo; t0 < hi; t0 += P2TILE) {
      long long kk[P2I];
#pragma unroll
      for (int q = 0; q < P2I; ++q) {
        const long long i = t0 + q * P2T + tid;
        kk[q] = i < hi ? (AOS ? stream_ld(&rec[i].k) : stream_ld(key + i)) : 0;
      }
#pragma unroll
      for (int q = 0; q < P2I; ++q)
        if (t0 + q * P2T + tid < hi)
          atomicAdd(&bins[g.logB2 ? (int)(((uint64_t)kk[q] >> (64 - g.logS)) & (nb2 - 1)) : 0],
                    1);
    }
    __syncthreads();
    for (int b = tid; b < nb2; b += P2T) hist[(long long)sg * nb2 + b] = bins[b];
  }
}

// Per sub-bucket (p, b), one thread: its rows, the sum of its count over the
// partition's segments.
__global__ void k_p2_colsum(const int* __restrict__ hist, const int* __restrict__ pseg, int S,
                            int logB2, long long* __restrict__ tot) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= S) return;
  const int p = idx >> logB2, b = idx & ((1 << logB2) - 1);
  const int nb2 = 1 << logB2;
  long long run = 0;
  for (int sg = pseg[p]; sg < pseg[p + 1]; ++sg) run += hist[(long long)sg * nb2 + b];
  tot[idx] = run;
}

// Region starts: cursor[i] = first[i] = i * cap for i < n.
__global__ void k_region_starts(unsigned long long* __restrict__ cursor,
                                unsigned long long* __restrict__ first, long long n,
                                long long cap) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long s = (unsigned long long)(i * cap);
    cursor[i] = s;
    if (first) first[i] = s;
  }
}

// After a first pass into regions, on the device (no host wait): per side
// and partition its start (p * cap) and rows (the cursor's advance, at most
// cap: a region that overflowed is cut at its end, and the overflow word
// makes the host run the pass again counted), into pstart ([2B] starts, then
// [2B] rows), and each partition's first second-pass tile into ts_b / ts_p
// ([B + 1], the last entry the side's tiles).  One block.
__global__ void __launch_bounds__(1024) k_pass1_plan(const unsigned long long* __restrict__ cur1,
                                                     int B, long long cap_b, long long cap_p,
                                                     long long tile_b, long long tile_p,
                                                     long long* __restrict__ pstart,
                                                     int* __restrict__ ts_b,
                                                     int* __restrict__ ts_p) {
  __shared__ long long wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int per = (B + 1023) / 1024;  // partitions a thread, consecutive
  for (int side = 0; side < 2; ++side) {
    const long long cap = side ? cap_p : cap_b, tile = side ? tile_p : tile_b;
    int* ts = side ? ts_p : ts_b;
    long long mine = 0;
    for (int j = 0; j < per; ++j) {
      const int p = tid * per + j;
      if (p >= B) break;
      const long long start = (long long)p * cap;
      const long long rows = min((long long)cur1[(size_t)side * B + p] - start, cap);
      pstart[(size_t)side * B + p] = start;
      pstart[2 * (size_t)B + (size_t)side * B + p] = rows;
      mine += (rows + tile - 1) / tile;
    }
    long long incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    long long pre = 0, total = 0;
    for (int q = 0; q < 32; ++q) {
      pre += q < w ? wsum[q] : 0;
      total += wsum[q];
    }
    long long run = pre + incl - mine;
    for (int j = 0; j < per; ++j) {
      const int p = tid * per + j;
      if (p >= B) break;
      ts[p] = (int)run;
      const long long rows = pstart[2 * (size_t)B + (size_t)side * B + p];
      run += (rows + tile - 1) / tile;
    }
    if (tid == 0) ts[B] = (int)total;
    __syncthreads();  // wsum is reused by the other side
  }
}

constexpr long long P2_SKIP = LLONG_MIN;  // a bin past its region: not written

template <int BINS, int TILE>
struct P2Smem {
  P2Row sr[TILE];
  int cnt[BINS];           // rows of a bin in the tile, then zero again
  int lofs[BINS];          // a bin's first place in the tile
  long long gpos[BINS];    // the bin's output place minus its tile place, or P2_SKIP
  int wsum[P2T / 32];
};

struct P2Args {
  const long long* key;     // MODE 1/2: raw keys; MODE 0 build: hashes
  const void* val;          // MODE 1 / MODE 0 build: int groups; MODE 2: int64 prices
  const long long* disc;    // MODE 2: discounts, or null (the value is the price)
  const P2Row* rec;         // MODE 0 probe: records
  long long n;              // MODE 1/2: rows
  long long scale;          // MODE 2: value = price * (scale - disc)
  const long long* pstart;  // MODE 0: each partition's first row
  const long long* pcnt;    // MODE 0: and rows
  const int* tstart;        // MODE 0: [B + 1] each partition's first tile
  int B;                    // MODE 0: partitions
  int logS, logB2;          // bins: the 2^logB2 hash bits below the top logS - logB2
  unsigned long long* cursor;  // per (sub-)bucket: its next free place
  long long cap;            // > 0: bin id's region ends at (id + 1) * cap
  unsigned long long* ovf;  // raised when a claim would cross its region's end
  long long* key_out;       // SoA outputs (build side)
  int* val_out;
  P2Row* rec_out;           // AoS output (probe side)
  // MODE 0 planned on the device: the first pass's overflow word; when it is
  // raised the partitions are cut short, so the probe side's pass does
  // nothing (the host runs everything again counted; the build side's pass,
  // a fifth of the work, runs regardless: the check would cost it registers)
  const unsigned long long* skip;
};

// Rows to their bin's run, tile by tile (so the blocks at work at one time
// all append to the same run ends, and each output line fills while it is in
// L2): each row's rank in its bin (a shared-memory atomic), the tile's
// exclusive scan over the bins, one claim per bin on its global cursor
// (travelling while the tile is staged in shared memory in bin order), then
// the write-out with consecutive threads on consecutive places (runs of about
// P2TILE / 2^logB2 rows).  The next tile's rows are loaded before the
// write-out.  Order inside a bin is not kept.  BULK (16-byte records, a
// 16-byte aligned output): each bin's run leaves shared memory as one TMA
// bulk copy issued by the thread that claimed it, instead of thread stores
// (measured on 600M probe rows: first pass 4.84 -> 4.37 ms, second pass
// 4.60 -> about 4.0).
//
// MODE 1 (first pass, build): rows (key, group) in row order, carried as
// (mix64(key), group), bins = the B buckets.  MODE 2 (first pass, probe): rows
// (fk, price, disc) carried as records (mix64(fk), price * (scale - disc)), or
// price when disc is null.  MODE 0 (second pass): tiles run partition by
// partition (tstart), the bins are the partition's 2^logB2 sub-buckets; the
// build side reads and writes (hash, group) columns, the probe side records.
// RI rows a thread a tile.
template <int MODE, bool AOS, int BINS, int RI, bool BULK>
__global__ void __launch_bounds__(P2T, PF_P2_MINB) k_p2_scatter(P2Args a) {
  using V = typename std::conditional<AOS, long long, int>::type;
  constexpr int BPT = BINS / P2T;
  constexpr int TILE = P2T * RI;
  constexpr int WU = PF_P2_WU;
  constexpr int LOGBINS = BINS == 4096 ? 12 : BINS == 2048 ? 11 : 10;
  static_assert(BINS == (1 << LOGBINS), "bins");
  static_assert(BULK == AOS, "records leave by bulk copies, columns by thread stores");
  extern __shared__ __align__(16) unsigned char p2_smem[];
  using Smem = P2Smem<BINS, TILE>;
  Smem& S = *reinterpret_cast<Smem*>(p2_smem);
  int* tps = reinterpret_cast<int*>(p2_smem + sizeof(Smem));  // MODE 0
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nb2 = 1 << a.logB2;
  const int bt = BPT * tid;  // the first of the bins this thread scans
#pragma unroll
  for (int j = 0; j < BPT; ++j) S.cnt[bt + j] = 0;
  long long ntiles;
  if (MODE == 0) {
    for (int p = tid; p <= a.B; p += P2T) tps[p] = a.tstart[p];
    __syncthreads();
    ntiles = AOS && a.skip && *a.skip ? 0 : tps[a.B];
  } else {
    ntiles = (a.n + TILE - 1) / TILE;
  }
  // tile t's rows [lo, hi) and its first bin's id
  auto locate = [&](long long t, long long& lo, long long& hi, long long& base) {
    if (MODE == 0) {
      int l = 0, r = a.B;  // tps[l] <= t < tps[r]: the last partition starting at or before t
      while (r - l > 1) {
        const int m = (l + r) >> 1;
        if (tps[m] <= t) l = m;
        else r = m;
      }
      const long long p0 = a.pstart[l];
      lo = p0 + (t - tps[l]) * TILE;
      hi = min(lo + TILE, p0 + a.pcnt[l]);
      base = (long long)l << a.logB2;
    } else {
      lo = t * TILE;
      hi = min(lo + TILE, a.n);
      base = 0;
    }
  };
  long long k[RI];
  V v[RI];
  // MODE 2 with a discount: the raw price in v and the discount in dv until
  // the tile's turn comes, so the prefetch never waits for its loads
  long long dv[MODE == 2 ? RI : 1];
  auto load = [&](long long lo, long long hi) {
#pragma unroll
    for (int q = 0; q < RI; ++q) {
      const long long i = lo + q * P2T + tid;
      if (i < hi) {
        if (MODE == 0 && AOS) {
          const P2Row r = stream_ld_row(a.rec + i);
          k[q] = r.k;
          v[q] = (V)r.v;
        } else {
          k[q] = stream_ld(a.key + i);
          v[q] = stream_ld(reinterpret_cast<const V*>(a.val) + i);
        }
        if (MODE == 2) dv[q] = a.disc ? stream_ld(a.disc + i) : 0;
      }
    }
  };
  long long tile = blockIdx.x;
  long long lo = 0, hi = 0, base = 0;
  if (tile < ntiles) {
    locate(tile, lo, hi, base);
    load(lo, hi);
  }
  __syncthreads();
  for (; tile < ntiles; tile += gridDim.x) {
#if PF_P2_L2PF
    // the rows of the tile after the next on their way into L2 (the next
    // one's are in flight into registers)
    if ((BULK || MODE == 1) && tid == 0 &&
        tile + PF_P2_L2PF * (long long)gridDim.x < ntiles) {
      long long plo, phi, pbase;
      locate(tile + PF_P2_L2PF * (long long)gridDim.x, plo, phi, pbase);
      const unsigned long long n = (unsigned long long)(phi - plo);
      if (MODE == 0 && AOS) {
        bulk_prefetch_l2(a.rec + plo, n * sizeof(P2Row));
      } else {
        bulk_prefetch_l2(a.key + plo, n * sizeof(long long));
        bulk_prefetch_l2(reinterpret_cast<const V*>(a.val) + plo, n * sizeof(V));
        if (MODE == 2 && a.disc) bulk_prefetch_l2(a.disc + plo, n * sizeof(long long));
      }
    }
#endif
    if (MODE != 0) {
#pragma unroll
      for (int q = 0; q < RI; ++q) k[q] = (long long)mix64((uint64_t)k[q]);
    }
    if (MODE == 2 && a.disc) {
#pragma unroll
      for (int q = 0; q < RI; ++q)
        v[q] = (V)(long long)((unsigned long long)v[q] * (unsigned long long)(a.scale - dv[q]));
    }
    // ranks from shared-memory adds, one a row (warp-match ranking, one add a
    // bin a warp after __match_any_sync, measured 1.5-1.9x slower on every
    // pass of the 150M x 600M join: few lanes of a warp share a bin here)
    int slot[RI];  // rank << LOGBINS | bin, or -1
#pragma unroll
    for (int q = 0; q < RI; ++q) {
      slot[q] = -1;
      if (lo + q * P2T + tid < hi) {
        const int b = MODE == 0 ? (a.logB2 ? (int)(((uint64_t)k[q] >> (64 - a.logS)) & (nb2 - 1)) : 0)
                                : bucket_of_hash((uint64_t)k[q], a.logS);
        slot[q] = (atomicAdd(&S.cnt[b], 1) << LOGBINS) | b;
      }
    }
    if (BULK) bulk_wait_read();  // the last tile's copies have read the staging
    __syncthreads();
    int cb[BPT];
    int s2 = 0;
#pragma unroll
    for (int j = 0; j < BPT; ++j) {
      cb[j] = S.cnt[bt + j];
      s2 += cb[j];
    }
    int incl = s2;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) S.wsum[w] = incl;
#pragma unroll
    for (int j = 0; j < BPT; ++j) S.cnt[bt + j] = 0;
    __syncthreads();
    int pre = 0, total = 0;
#pragma unroll
    for (int q = 0; q < P2T / 32; ++q) {
      const int x = S.wsum[q];
      pre += q < w ? x : 0;
      total += x;
    }
    int lofs[BPT];
    {
      int run = pre + incl - s2;
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        lofs[j] = run;
        S.lofs[bt + j] = run;
        run += cb[j];
      }
    }
    __syncthreads();
    // the claims travel while the tile is placed (issued right after the
    // counts instead: no faster)
    long long gp[BPT];
#pragma unroll
    for (int j = 0; j < BPT; ++j)
      gp[j] = cb[j] ? (long long)atomicAdd(&a.cursor[base + bt + j], (unsigned long long)cb[j]) : 0;
    // every row's tile place first (the loads overlap), then the stores
#pragma unroll
    for (int q = 0; q < RI; ++q)
      if (slot[q] >= 0) slot[q] = S.lofs[slot[q] & (BINS - 1)] + (slot[q] >> LOGBINS);
#pragma unroll
    for (int q = 0; q < RI; ++q)
      if (slot[q] >= 0) S.sr[slot[q]] = P2Row{k[q], (long long)v[q]};
    // per bin, its output place minus its first place in the tile (a row at
    // tile place e goes to e + that), or the skip mark
#pragma unroll
    for (int j = 0; j < BPT; ++j) {
      long long d = gp[j] - lofs[j];
      if (a.cap > 0 && cb[j] && gp[j] + cb[j] > (base + bt + j + 1) * a.cap) {
        *a.ovf = 1;  // past the region: none of the bin's rows are written
        d = P2_SKIP;
      }
      S.gpos[bt + j] = d;
    }
    if (BULK) fence_proxy_async_smem();  // the staged rows, to the bulk copies
    __syncthreads();
    const long long base_cur = base;
    if (tile + gridDim.x < ntiles) {
      locate(tile + gridDim.x, lo, hi, base);
      load(lo, hi);
    }
    if constexpr (BULK) {
      // each bin's staged run to its claimed place with one bulk copy
      // (records of 16 bytes: both ends 16-byte aligned); the staging is
      // reused only after every copy of this tile has read it (the wait
      // before the next tile's first barrier)
      bool issued = false;
#pragma unroll
      for (int j = 0; j < BPT; ++j) {
        if (!cb[j]) continue;
        if (a.cap > 0 && gp[j] + cb[j] > (base_cur + bt + j + 1) * a.cap) continue;
        bulk_s2g(a.rec_out + gp[j], &S.sr[lofs[j]], (unsigned)cb[j] * (unsigned)sizeof(P2Row));
        issued = true;
      }
      if (issued) bulk_commit();
    } else {
      // WU staged rows a thread at a time: their loads, then their bins'
      // places, then their stores
      for (int e0 = tid; e0 < total; e0 += P2T * WU) {
        P2Row r[WU];
        long long d[WU];
#pragma unroll
        for (int u = 0; u < WU; ++u)
          if (e0 + u * P2T < total) r[u] = S.sr[e0 + u * P2T];
#pragma unroll
        for (int u = 0; u < WU; ++u) {
          d[u] = P2_SKIP;
          if (e0 + u * P2T < total) {
            const int b =
                MODE == 0 ? (a.logB2 ? (int)(((uint64_t)r[u].k >> (64 - a.logS)) & (nb2 - 1)) : 0)
                          : bucket_of_hash((uint64_t)r[u].k, a.logS);
            d[u] = S.gpos[b];
          }
        }
#pragma unroll
        for (int u = 0; u < WU; ++u) {
          if (d[u] == P2_SKIP) continue;
          const long long pos = d[u] + e0 + u * P2T;
          a.key_out[pos] = r[u].k;
          a.val_out[pos] = (int)r[u].v;
        }
      }
    }
    // no barrier here: the next tile's ranking touches only the counts
    // (zeroed before this tile's second barrier), and its first barrier
    // waits for every thread's write-out before the staging is reused
  }
  if (BULK) bulk_wait_all();
}

struct SJArgs {
  const long long* bkey;
  const int* bgrp;
  const P2Row* prec;
  const unsigned long long* bbeg;  // [S]: each sub-partition's build rows [bbeg, bend)
  const unsigned long long* bend;
  const unsigned long long* pbeg;  // and probe rows [pbeg, pend)
  const unsigned long long* pend;
  long long S;
  int logS;
  long long group_min, n_groups;
  unsigned long long* slab;
  unsigned long long* stats;
  unsigned long long* counter;
  const unsigned long long* ovf;   // nonzero: a region overflowed, nothing to join
  const unsigned long long* ovf1;  // and the first pass's, when its plan was made on the device
};

// A cell's 64-bit sum in shared memory as two 32-bit words, each in an array
// of its own (a warp's random cells then spread over all 32 banks), added with
// 32-bit atomics: the low word's add returns its old value, which shows the
// carry into the high word (measured against one 64-bit shared add: 4.39
// against 5.08 ms for the 150M x 600M join).
struct SJSmem {
  long long key[SJ_TS];
  unsigned sum_lo[SJ_TS];
  unsigned sum_hi[SJ_TS];
  unsigned cnt[SJ_TS];
  unsigned short slot_of[SJ_CAP];  // the slot of each build row of the chunk
  long long min_sum;               // the key hashing to INT64_MIN, kept apart
  unsigned min_cnt, min_goff;
  int has_min;
  long long item[2];               // sub-partition and its row ranges, double-buffered
  long long bnd[2][4];
};

__device__ __forceinline__ void sj_sum_add(SJSmem& S, unsigned t, long long val) {
  const unsigned l = (unsigned)(unsigned long long)val;
  const unsigned h = (unsigned)((unsigned long long)val >> 32);
  const unsigned old = atomicAdd(&S.sum_lo[t], l);
  const unsigned hc = h + (old + l < old ? 1u : 0u);
  if (hc) atomicAdd(&S.sum_hi[t], hc);  // zero for a value below 2^32 without a carry
}
__device__ __forceinline__ unsigned long long sj_sum_get(const SJSmem& S, unsigned t) {
  return ((unsigned long long)S.sum_hi[t] << 32) | S.sum_lo[t];
}
__device__ __forceinline__ void sj_sum_clear(SJSmem& S, unsigned t) {
  S.sum_lo[t] = 0;
  S.sum_hi[t] = 0;
}

// A row's home slot: the PF_SJ_LOGTS hash bits after the top logS ones (which
// all rows of a sub-partition share); from the high word alone when they lie
// in it.
__device__ __forceinline__ unsigned sj_slot(uint64_t h, int logS) {
  if (!SJ_POW2)  // the next 32 bits scaled onto the slots
    return (unsigned)(((unsigned long long)(unsigned)((h << logS) >> 32) * SJ_TS) >> 32);
  if (logS + PF_SJ_LOGTS <= 32) return ((unsigned)(h >> 32) << logS) >> (32 - PF_SJ_LOGTS);
  return (unsigned)((h << logS) >> (64 - PF_SJ_LOGTS));
}
__device__ __forceinline__ unsigned sj_next(unsigned t) {
  return SJ_POW2 ? (t + 1) & (SJ_TS - 1) : (t + 1 == (unsigned)SJ_TS ? 0u : t + 1);
}

// One probe row against the chunk's table: its value and 1 into the cell of
// the build row with its key.
__device__ __forceinline__ void sj_probe(SJSmem& S, long long key, long long val, int logS,
                                         unsigned& matched) {
  if (key == SJ_EMPTY) {
    if (S.has_min) {
      atomicAdd((unsigned long long*)&S.min_sum, (unsigned long long)val);
      atomicAdd(&S.min_cnt, 1u);
      ++matched;
    }
    return;
  }
  unsigned t = sj_slot((uint64_t)key, logS);
  for (int probes = 0; probes < SJ_TS; ++probes) {
    const long long x = S.key[t];
    if (x == SJ_EMPTY) return;
    if (x == key) {
      sj_sum_add(S, t, val);
      atomicAdd(&S.cnt[t], 1u);
      ++matched;
      return;
    }
    t = sj_next(t);
  }
}

__global__ void __launch_bounds__(SJT, PF_SJ_MINB) k_sjoin(SJArgs a) {
  extern __shared__ __align__(16) unsigned char sj_smem[];
  SJSmem& S = *reinterpret_cast<SJSmem*>(sj_smem);
  // the partitions are incomplete: the host runs the counted passes
  if (*a.ovf || (a.ovf1 && *a.ovf1)) return;
  const int tid = threadIdx.x;
  for (int t = tid; t < SJ_TS; t += SJT) {
    S.key[t] = SJ_EMPTY;
    sj_sum_clear(S, t);
    S.cnt[t] = 0;
  }
  unsigned matched = 0;  // rows a thread matched (below 2^32: at most 2^40 / SJT)
  unsigned bad_group = 0;  // below 2^32: a thread flushes at most 2^40 / SJT rows
  // Thread 0 fetches the next sub-partition and its ranges into the other
  // half of a double-buffered descriptor while the block works on the
  // current one; the barriers of the work make it visible.
  auto fetch = [&](int slot) {
    const long long n = (long long)atomicAdd(a.counter, 1ULL);
    S.item[slot] = n;
    if (n < a.S) {
      S.bnd[slot][0] = (long long)a.bbeg[n];
      S.bnd[slot][1] = (long long)a.bend[n];
      S.bnd[slot][2] = (long long)a.pbeg[n];
      S.bnd[slot][3] = (long long)a.pend[n];
    }
  };
  if (tid == 0) {
    S.has_min = 0;
    S.min_sum = 0;
    S.min_cnt = 0;
    fetch(0);
  }
  __syncthreads();
  for (int cur = 0;; cur ^= 1) {
    const long long s = S.item[cur];
    const long long b0 = S.bnd[cur][0], b1 = S.bnd[cur][1];
    const long long p0 = S.bnd[cur][2], p1 = S.bnd[cur][3];
    if (s >= a.S) break;
    if (tid == 0) fetch(cur ^ 1);
    if (b1 <= b0 || p1 <= p0) {
      __syncthreads();
      continue;
    }
    for (long long c0 = b0; c0 < b1; c0 += SJ_CAP) {
      const int nb = (int)min((long long)SJ_CAP, b1 - c0);
#if PF_SJ_PIPE
      // the first probe round's rows load while the build runs; pr walks
      // this thread's rows (every SJT-th from p0 + tid), rem counts the rows
      // from the current one to the end of the range
      const P2Row* pr = a.prec + p0 + tid;
      const long long rem = p1 - p0 - tid;
      P2Row row[SJ_U];
#pragma unroll
      for (int u = 0; u < SJ_U; ++u) row[u] = u * SJT < rem ? stream_ld_row(pr + u * SJT) : P2Row{0, 0};
#endif
      // build: each build row a slot of its own (all of a thread's rows
      // loaded first)
      // (and their groups, held until the flush: measured 0.18 ms less than
      // reading them again there)
      long long bk[SJ_BU];
      int bg[SJ_BU];
#pragma unroll
      for (int u = 0; u < SJ_BU; ++u) {
        const int j = u * SJT + tid;
        if (j < nb) {
          bk[u] = stream_ld(a.bkey + c0 + j);
          bg[u] = stream_ld(a.bgrp + c0 + j);
        }
      }
#pragma unroll
      for (int u = 0; u < SJ_BU; ++u) {
        if (u * SJT + tid >= nb) continue;
        const long long key = bk[u];
        if (key == SJ_EMPTY) {
          const long long g = (long long)a.bgrp[c0 + u * SJT + tid] - a.group_min;
          S.has_min = 1;
          S.min_goff = g >= 0 && g < a.n_groups ? (unsigned)g : SJ_NONE;
          S.slot_of[u * SJT + tid] = 0xffff;
          continue;
        }
        unsigned t = sj_slot((uint64_t)key, a.logS);
        for (int probes = 0; probes < SJ_TS; ++probes) {
          const long long old = (long long)atomicCAS((unsigned long long*)&S.key[t],
                                                     (unsigned long long)SJ_EMPTY,
                                                     (unsigned long long)key);
          if (old == SJ_EMPTY) break;
          t = sj_next(t);
        }
        S.slot_of[u * SJT + tid] = (unsigned short)t;
      }
      __syncthreads();
      // probe, SJ_U rows a thread a round
#if PF_SJ_PIPE
      // the next round's rows load while this round's are looked up
      {
        P2Row nrow[SJ_U];
        constexpr int STEP = SJT * SJ_U;
        for (long long r = rem; r > 0; r -= STEP) {
          pr += STEP;
          const long long rn = r - STEP;
#pragma unroll
          for (int u = 0; u < SJ_U; ++u)
            nrow[u] = u * SJT < rn ? stream_ld_row(pr + u * SJT) : P2Row{0, 0};
#pragma unroll
          for (int u = 0; u < SJ_U; ++u)
            if (u * SJT < r) sj_probe(S, row[u].k, row[u].v, a.logS, matched);
#pragma unroll
          for (int u = 0; u < SJ_U; ++u) row[u] = nrow[u];
        }
      }
#else
      for (long long i0 = p0; i0 < p1; i0 += (long long)SJT * SJ_U) {
        P2Row row[SJ_U];
#pragma unroll
        for (int u = 0; u < SJ_U; ++u) {
          const long long i = i0 + u * SJT + tid;
          if (i < p1) row[u] = stream_ld_row(a.prec + i);
        }
#pragma unroll
        for (int u = 0; u < SJ_U; ++u)
          if (i0 + u * SJT + tid < p1) sj_probe(S, row[u].k, row[u].v, a.logS, matched);
      }
#endif
      __syncthreads();
      // flush every build row that matched (the thread's own build rows,
      // their groups in registers), and empty its slot
#pragma unroll
      for (int u = 0; u < SJ_BU; ++u) {
        const int j = u * SJT + tid;
        if (j >= nb) continue;
        const unsigned t = S.slot_of[j];
        if (t == 0xffff) continue;
        const unsigned c = S.cnt[t];
        const long long g = (long long)bg[u] - a.group_min;
        const bool gok = g >= 0 && g < a.n_groups;
        bad_group += !gok;
        if (c && gok) {
          atomicAdd(&a.slab[2 * (unsigned long long)g], sj_sum_get(S, t));
          atomicAdd(&a.slab[2 * (unsigned long long)g + 1], (unsigned long long)c);
        }
        S.key[t] = SJ_EMPTY;
        sj_sum_clear(S, t);
        S.cnt[t] = 0;
      }
      if (tid == 0) {
        if (S.has_min) {
          bad_group += S.min_goff == SJ_NONE;
          if (S.min_cnt && S.min_goff != SJ_NONE) {
            atomicAdd(&a.slab[2 * (unsigned long long)S.min_goff], (unsigned long long)S.min_sum);
            atomicAdd(&a.slab[2 * (unsigned long long)S.min_goff + 1],
                      (unsigned long long)S.min_cnt);
          }
        }
        S.has_min = 0;
        S.min_sum = 0;
        S.min_cnt = 0;
      }
      __syncthreads();
    }
  }
  unsigned long long m = matched;
  for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(FULL, m, o);
  if ((tid & 31) == 0 && m) atomicAdd(&a.stats[0], m);
  if (bad_group) atomicAdd(&a.stats[2], (unsigned long long)bad_group);
}

// ---- the join with a fingerprinted slot table ----------------------------------
//
// The same join per sub-partition with the table split in three: 4-byte
// slots {build row + 1 (11 bits) | fingerprint (21 low hash bits)}, 0 = free,
// at a load of at most 0.375; the chunk's build hashes by row; and the cells
// (sum as two 32-bit words, count) by row.  A probe row walks slots until a
// free one, reading a build row's hash only where the fingerprint agrees.
// 4-byte slots let the table be larger for the same shared memory (shorter
// walks, fewer divergent lanes), the cells are flushed in row order, and no
// hash value is reserved as a free mark.
#ifndef PF_SJF_LOGTS
#define PF_SJF_LOGTS 12
#endif
#ifndef PF_SJF_T
#define PF_SJF_T 384
#endif
#ifndef PF_SJF_MINB
#define PF_SJF_MINB 4
#endif
constexpr int SJF_TS = 1 << PF_SJF_LOGTS;   // slots
constexpr int SJF_T = PF_SJF_T;              // threads
constexpr int SJF_CAP = 1536;                // build rows a chunk (row + 1 fits 11 bits)
constexpr int SJF_BU = (SJF_CAP + SJF_T - 1) / SJF_T;
constexpr unsigned SJF_FPBITS = 21;
constexpr unsigned SJF_FPMASK = (1u << SJF_FPBITS) - 1;
static_assert(SJF_CAP < (1 << (32 - SJF_FPBITS)), "row + 1 fits the slot's high bits");
static_assert(SJF_CAP * 8 <= SJF_TS * 3, "load at most 0.375");

struct SJFSmem {
  unsigned slot[SJF_TS];
  long long bh[SJF_CAP];           // the chunk's build hashes by row
  unsigned lo[SJF_CAP], hi[SJF_CAP], cnt[SJF_CAP];
  unsigned short slot_of[SJF_CAP]; // each build row's slot (to free it)
  long long item[2];               // sub-partition and its row ranges, double-buffered
  long long bnd[2][4];
};

__device__ __forceinline__ unsigned sjf_home(uint64_t h, int logS) {
  if (logS + PF_SJF_LOGTS <= 32) return ((unsigned)(h >> 32) << logS) >> (32 - PF_SJF_LOGTS);
  return (unsigned)((h << logS) >> (64 - PF_SJF_LOGTS));
}

__global__ void __launch_bounds__(SJF_T, PF_SJF_MINB) k_sjoin_fp(SJArgs a) {
  extern __shared__ __align__(16) unsigned char sjf_smem[];
  SJFSmem& S = *reinterpret_cast<SJFSmem*>(sjf_smem);
  if (*a.ovf || (a.ovf1 && *a.ovf1)) return;  // the partitions are incomplete: the host runs the counted passes
  const int tid = threadIdx.x;
  for (int t = tid; t < SJF_TS; t += SJF_T) S.slot[t] = 0;
  for (int r = tid; r < SJF_CAP; r += SJF_T) {
    S.lo[r] = 0;
    S.hi[r] = 0;
    S.cnt[r] = 0;
  }
  unsigned matched = 0;
  unsigned long long bad_group = 0;
  auto fetch = [&](int slot) {
    const long long n = (long long)atomicAdd(a.counter, 1ULL);
    S.item[slot] = n;
    if (n < a.S) {
      S.bnd[slot][0] = (long long)a.bbeg[n];
      S.bnd[slot][1] = (long long)a.bend[n];
      S.bnd[slot][2] = (long long)a.pbeg[n];
      S.bnd[slot][3] = (long long)a.pend[n];
    }
  };
  if (tid == 0) fetch(0);
  __syncthreads();
  for (int cur = 0;; cur ^= 1) {
    const long long s = S.item[cur];
    const long long b0 = S.bnd[cur][0], b1 = S.bnd[cur][1];
    const long long p0 = S.bnd[cur][2], p1 = S.bnd[cur][3];
    if (s >= a.S) break;
    if (tid == 0) fetch(cur ^ 1);
    if (b1 <= b0 || p1 <= p0) {
      __syncthreads();
      continue;
    }
    for (long long c0 = b0; c0 < b1; c0 += SJF_CAP) {
      const int nb = (int)min((long long)SJF_CAP, b1 - c0);
      // the first probe round's rows load while the build runs
      const P2Row* pr = a.prec + p0 + tid;
      const long long rem = p1 - p0 - tid;
      P2Row row = rem > 0 ? stream_ld_row(pr) : P2Row{0, 0};
      long long bk[SJF_BU];
#pragma unroll
      for (int u = 0; u < SJF_BU; ++u) {
        const int j = u * SJF_T + tid;
        if (j < nb) bk[u] = stream_ld(a.bkey + c0 + j);
      }
#pragma unroll
      for (int u = 0; u < SJF_BU; ++u) {
        const int j = u * SJF_T + tid;
        if (j >= nb) continue;
        const uint64_t h = (uint64_t)bk[u];
        S.bh[j] = (long long)h;
        const unsigned e = ((unsigned)(j + 1) << SJF_FPBITS) | ((unsigned)h & SJF_FPMASK);
        unsigned t = sjf_home(h, a.logS);
        for (int probes = 0; probes < SJF_TS; ++probes) {
          if (atomicCAS(&S.slot[t], 0u, e) == 0u) break;
          t = (t + 1) & (SJF_TS - 1);
        }
        S.slot_of[j] = (unsigned short)t;
      }
      __syncthreads();
      // probe: the next round's row loads while this one's is looked up
      for (long long r = rem; r > 0; r -= SJF_T) {
        pr += SJF_T;
        const P2Row next = r > SJF_T ? stream_ld_row(pr) : P2Row{0, 0};
        const uint64_t h = (uint64_t)row.k;
        const unsigned fp = (unsigned)h & SJF_FPMASK;
        unsigned t = sjf_home(h, a.logS);
        for (int probes = 0; probes < SJF_TS; ++probes) {
          const unsigned e = S.slot[t];
          if (e == 0u) break;
          if ((e & SJF_FPMASK) == fp) {
            const int j = (int)(e >> SJF_FPBITS) - 1;
            if ((uint64_t)S.bh[j] == h) {
              const unsigned l = (unsigned)(unsigned long long)row.v;
              const unsigned hw = (unsigned)((unsigned long long)row.v >> 32);
              const unsigned old = atomicAdd(&S.lo[j], l);
              const unsigned hc = hw + (old + l < old ? 1u : 0u);
              if (hc) atomicAdd(&S.hi[j], hc);
              atomicAdd(&S.cnt[j], 1u);
              ++matched;
              break;
            }
          }
          t = (t + 1) & (SJF_TS - 1);
        }
        row = next;
      }
      __syncthreads();
      // flush every build row that matched (its group read again, from L2),
      // and free its slot and cell
      for (int j = tid; j < nb; j += SJF_T) {
        const unsigned c = S.cnt[j];
        const long long g = (long long)a.bgrp[c0 + j] - a.group_min;
        const bool gok = g >= 0 && g < a.n_groups;
        bad_group += !gok;
        if (c && gok) {
          atomicAdd(&a.slab[2 * (unsigned long long)g],
                    ((unsigned long long)S.hi[j] << 32) | S.lo[j]);
          atomicAdd(&a.slab[2 * (unsigned long long)g + 1], (unsigned long long)c);
        }
        S.slot[S.slot_of[j]] = 0;
        S.lo[j] = 0;
        S.hi[j] = 0;
        S.cnt[j] = 0;
      }
      __syncthreads();
    }
  }
  unsigned long long m = matched;
  for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(FULL, m, o);
  if ((tid & 31) == 0 && m) atomicAdd(&a.stats[0], m);
  if (bad_group) atomicAdd(&a.stats[2], bad_group);
}

// The run-time choices of one call (pf_join_knobs with the defaults filled
// in): the join path, the shared-memory join's table, the build rows a
// sub-partition aims at, and whether the radix passes count first.  Without
// knobs from the caller, PF_JOIN_PATH=rounds|smem, PF_SJ_FP=0|1,
// PF_SJ_TARGET=<rows> and PF_COUNTED=0|1 override the defaults (sweeps and
// tests); the workspace depends on them, so a query and its call must see
// the same ones.
struct Knobs {
  int smem;          // 1: the shared-memory join, 0: the L2-round join
  int table;         // shared-memory join: 0 hash slots, 1 fingerprinted slots
  long long target;  // build rows a sub-partition aims at
  int counted;       // 1: both radix passes count their rows first
};

Knobs resolve_knobs(const pf_join_knobs* k) {
  Knobs r{PF_JOIN_PATH_DEFAULT, PF_SJ_FP_DEFAULT, SJ_TARGET, 0};
  if (k) {
    r.smem = k->path == 0 ? 1 : 0;
    r.table = k->table ? 1 : 0;
    if (k->sub_rows > 0) r.target = k->sub_rows;
    r.counted = k->counted ? 1 : 0;
    return r;
  }
  if (const char* e = getenv("PF_JOIN_PATH")) {
    if (std::string(e) == "rounds") r.smem = 0;
    if (std::string(e) == "smem") r.smem = 1;
  }
  if (const char* e = getenv("PF_SJ_FP")) r.table = e[0] == '1';
  if (const char* e = getenv("PF_SJ_TARGET")) r.target = std::max(64LL, atoll(e));
  if (const char* e = getenv("PF_COUNTED")) r.counted = e[0] == '1';
  return r;
}

// The interleaved slab split into the caller's sum and count arrays.
__global__ void k_split(const unsigned long long* __restrict__ slab, long long n,
                        long long* __restrict__ sum, long long* __restrict__ count) {
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const ulonglong2 v = reinterpret_cast<const ulonglong2*>(slab)[g];
    sum[g] = (long long)v.x;
    count[g] = (long long)v.y;
  }
}

// The regions of the rounds, from the build counts: the same greedy packing
// as the host's plan (one thread; B <= 4096).  A partition over the budget
// gets no region here (its slice rounds pass their own).
__global__ void k_plan(const long long* __restrict__ cnt, int B, long long cap_rows,
                       long long* __restrict__ reg) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  long long rows = 0;
  for (int p = 0; p < B; ++p) {
    const long long n = cnt[p];
    if (n > cap_rows) {
      reg[p] = 0;
      reg[B + p] = 0;
      rows = 0;
      continue;
    }
    if (rows + n > cap_rows) rows = 0;
    reg[p] = 2 * rows;
    reg[B + p] = 2 * n;
    rows += n;
  }
}

// ---- finish: the groups present, ascending ------------------------------------------

__global__ void __launch_bounds__(CT) k_gcount(const long long* __restrict__ count, long long n,
                                               long long* __restrict__ bcnt) {
  const long long base = (long long)blockIdx.x * CB;
  int c = 0;
  for (int k = 0; k < CITEMS; ++k) {
    const long long i = base + k * CT + threadIdx.x;
    if (i < n) c += count[i] > 0;
  }
  __shared__ int red[CT / 32];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int q = 0; q < CT / 32; ++q) t += red[q];
    bcnt[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(CT) k_gemit(const long long* __restrict__ sum,
                                              const long long* __restrict__ count, long long n,
                                              long long group_min,
                                              const long long* __restrict__ boff,
                                              long long* __restrict__ keys,
                                              long long* __restrict__ sums,
                                              long long* __restrict__ counts) {
  __shared__ int wsum[CT / 32];
  const long long base = (long long)blockIdx.x * CB + (long long)threadIdx.x * CITEMS;
  bool kp[CITEMS];
  int rank[CITEMS];
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) kp[k] = base + k < n && count[base + k] > 0;
  __shared__ unsigned short rows[CB];
  const int tot = block_compact(kp, rank, rows, wsum);
  const long long o = boff[blockIdx.x], b0 = (long long)blockIdx.x * CB;
  for (int e = threadIdx.x; e < tot; e += CT) {
    const long long r = b0 + rows[e];
    keys[o + e] = group_min + r;
    sums[o + e] = sum[r];
    counts[o + e] = count[r];
  }
}

// ---- host ------------------------------------------------------------------------------

long long round_rows() {
  static long long v = [] {
    const char* e = getenv("PF_ROUND_ROWS");
    long long x = e ? atoll(e) : 0;
    return x > 0 ? x : ROUND_ROWS_DEFAULT;
  }();
  return v;
}

#ifndef PF_CHUNKS_PER_SM
#define PF_CHUNKS_PER_SM 2
#endif

void chunking(long long n, long long* chunk, int* nchunks) {
  const long long subs = std::max<long long>(1, (n + FSUB - 1) / FSUB);
  const long long want = std::max<long long>(1, (long long)sm_count() * PF_CHUNKS_PER_SM);
  const long long per = (subs + want - 1) / want;
  *chunk = per * FSUB;
  *nchunks = (int)std::max<long long>(1, (n + *chunk - 1) / *chunk);
}

// The passes the calling thread's last call counted first (bit 0: first, bit 1:
// second).
thread_local int g_counted_passes = 0;

struct JaLayout {
  int* hist_b;
  int* hist_p;
  long long* cnt;      // [2B]: build counts, probe counts
  long long* start;    // [2B]: build starts, probe starts
  long long* total;    // [2]
  long long* pkey;     // the first pass's build side (hash or key, group)
  int* pgrp;
  long long* pfk;      // the round path's probe side (key, value)
  long long* pval;
  Slot* table;
  long long table_slots;
  long long* reg;      // [2B]: reg_off, reg_cap
  unsigned long long* slab;  // [2 * n_groups]: (sum, count) per group
  long long max_launches;
  unsigned* counters;        // [max_launches] work counters of the round launches
  // the shared-memory path
  long long cap1[2];         // rows of a first-pass bucket's region, per side
  P2Row* prec;               // the first pass's probe side (records)
  long long s_max;           // sub-partitions at most
  long long rows2[2];        // rows of the second pass's output, per side
  long long* pkey2;
  int* pgrp2;
  P2Row* prec2;
  long long* pstart;         // [2B]: each side's partition starts, then [2B] rows
  int* tstart[2];            // [B + 1]: each partition's first second-pass tile
  long long nseg_max[2];     // counted second pass: segments a side, at most
  int2* seg2[2];             // the segments of each side
  int* pseg2[2];             // [B + 1]: each partition's first segment
  int* hist2[2];             // [segments][2^logB2]
  unsigned long long* cur2;    // [2][s_max]: the second pass's cursors
  unsigned long long* beg2;    // [2][s_max]: its regions' starts
  unsigned long long* cur1;    // [2B]: the first pass's cursors
  long long* tot2;             // [2][s_max]: rows per sub-partition (counted)
  unsigned long long* start2;  // [2][s_max + 1]
  long long* scan2;            // scan scratch
  unsigned long long* sj_counter;
  unsigned long long* ovf;     // [2]: a region of the first / second pass overflowed
};

// Sub-partitions a partition splits into at most (a power of two): never
// finer than `target` build rows.
long long max_subparts(long long nb, long long target) {
  return std::min<long long>(P2BINS, (long long)pow2_at_least((uint64_t)(nb / target + 1)));
}

// The second radix pass's and the join's share of the workspace, for nparts
// partitions of at most maxp[side] rows: regions for partitions that full,
// the plan of the counted pass, the join's counter.
void take_second_pass(Arena& a, JaLayout& l, long long nb, long long np, int nparts,
                      const long long maxp[2], long long target) {
  const long long rows[2] = {nb, np};
  const long long b2 = max_subparts(std::max(maxp[0], nb / std::max(1, nparts)), target);
  l.s_max = (long long)nparts * b2;
  for (int side = 0; side < 2; ++side)
    l.rows2[side] = std::max(std::max<long long>(rows[side], 1),
                             l.s_max * region_rows((double)maxp[side] / b2, region_var(side)));
  l.pkey2 = a.take<long long>((size_t)l.rows2[0]);
  l.pgrp2 = a.take<int>((size_t)l.rows2[0]);
  l.prec2 = a.take<P2Row>((size_t)l.rows2[1]);
  l.pstart = a.take<long long>(4 * (size_t)nparts);
  for (int side = 0; side < 2; ++side) {
    l.tstart[side] = a.take<int>((size_t)nparts + 1);
    l.nseg_max[side] = rows[side] / P2SEG + nparts + 1;
    l.seg2[side] = a.take<int2>((size_t)l.nseg_max[side]);
    l.pseg2[side] = a.take<int>((size_t)nparts + 1);
    l.hist2[side] = a.take<int>((size_t)l.nseg_max[side] * P2BINS);
  }
  l.tot2 = a.take<long long>(2 * (size_t)l.s_max);
  l.cur2 = a.take<unsigned long long>(2 * (size_t)l.s_max);
  l.beg2 = a.take<unsigned long long>(2 * (size_t)l.s_max);
  l.start2 = a.take<unsigned long long>(2 * ((size_t)l.s_max + 1));
  l.scan2 = a.take<long long>(scan_scratch_elems(l.s_max));
  l.sj_counter = a.take<unsigned long long>(1);
}

JaLayout ja_layout(Arena& a, long long nb, long long np, int B, long long n_groups,
                   const Knobs& kn) {
  JaLayout l{};
  long long chunk;
  int nb_ch, np_ch;
  chunking(nb, &chunk, &nb_ch);
  chunking(np, &chunk, &np_ch);
  l.hist_b = a.take<int>((size_t)nb_ch * B);
  l.hist_p = a.take<int>((size_t)np_ch * B);
  l.cnt = a.take<long long>(2 * (size_t)B);
  l.start = a.take<long long>(2 * (size_t)B);
  l.total = a.take<long long>(2);
  l.reg = a.take<long long>(2 * (size_t)B);
  l.slab = a.take<unsigned long long>(2 * (size_t)std::max<long long>(n_groups, 1));
  l.ovf = a.take<unsigned long long>(2);
  if (!kn.smem) {
    l.pkey = a.take<long long>(std::max<long long>(nb, 1));
    l.pgrp = a.take<int>(std::max<long long>(nb, 1));
    l.pfk = a.take<long long>(std::max<long long>(np, 1));
    l.pval = a.take<long long>(std::max<long long>(np, 1));
    // two halves, one built while the other is probed
    l.table_slots = 2 * std::max<long long>(1, std::min(nb, round_rows()));
    l.table = a.take<Slot>(2 * l.table_slots);
    // one work counter per launch: at most B whole-partition rounds plus the
    // slices of partitions over the budget, plus one
    l.max_launches = B + nb / std::max<long long>(1, l.table_slots / 2) + 2;
    l.counters = a.take<unsigned>(l.max_launches);
    return l;
  }
  // first pass: a region of cap1 rows a bucket (at least the side's rows)
  const long long rows[2] = {nb, np};
  for (int side = 0; side < 2; ++side)
    l.cap1[side] = std::max((rows[side] + B - 1) / B,
                            region_rows((double)rows[side] / B, region_var(side)));
  l.pkey = a.take<long long>((size_t)B * l.cap1[0]);
  l.pgrp = a.take<int>((size_t)B * l.cap1[0]);
  l.prec = a.take<P2Row>((size_t)B * l.cap1[1]);
  take_second_pass(a, l, nb, np, B, l.cap1, kn.target);
  l.cur1 = a.take<unsigned long long>(2 * (size_t)B);
  return l;
}

struct Round {
  int p0, p1;            // partitions [p0, p1)
  long long b_lo, b_hi;  // build rows
  long long p_lo, p_hi;  // probe rows
  long long slice_cap;   // > 0: one slice of partition p0
};

// A thread's pinned staging buffer for the bucket counts.
long long* pinned_counts(size_t n) {
  thread_local long long* buf = nullptr;
  thread_local size_t have = 0;
  if (have < n) {
    if (buf) cudaFreeHost(buf);
    buf = nullptr;
    have = 0;
    if (cudaHostAlloc((void**)&buf, n * sizeof(long long), cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    have = n;
  }
  return buf;
}


// The round path's first radix pass of both sides (the TMA-fed kernel when
// every column is 16-byte aligned).
int fscatter_rounds(bool tma, const int64_t* build_key, const int32_t* build_group,
                    long long n_build, const int64_t* probe_fk, const int64_t* probe_price,
                    const int64_t* probe_disc, long long scale, long long n_probe,
                    long long chunk_b, int nch_b, long long chunk_p, int nch_p, int logB, int B,
                    const JaLayout& l, int64_t* stats_out, cudaStream_t st) {
  if (tma) {
    const size_t smb = tma_smem<false>(B), smp = tma_smem<true>(B);
    if (int rc = opt_in_smem((const void*)k_fscatter_tma<false, false>, smb)) return rc;
    if (int rc = opt_in_smem((const void*)k_fscatter_tma<true, false>, smp)) return rc;
    {
      PF_KERNEL("k_fscatter_build", st);
      k_fscatter_tma<false, false><<<nch_b, TT, smb, st>>>(
          (const long long*)build_key, build_group, nullptr, 0, n_build, chunk_b, logB, B,
          tma_nbuf<false>(B), l.hist_b, l.start, l.pkey, l.pgrp, (unsigned long long*)stats_out + 1);
    }
    {
      PF_KERNEL("k_fscatter_probe", st);
      k_fscatter_tma<true, false><<<nch_p, TT, smp, st>>>(
          (const long long*)probe_fk, probe_price, (const long long*)probe_disc, scale, n_probe,
          chunk_p, logB, B, tma_nbuf<true>(B), l.hist_p, l.start + B, l.pfk, l.pval,
          (unsigned long long*)stats_out + 1);
    }
  } else {
    const size_t smb = fscatter_smem(B, false), smp = fscatter_smem(B, true);
    if (int rc = opt_in_smem((const void*)k_fscatter<false, false>, smb)) return rc;
    if (int rc = opt_in_smem((const void*)k_fscatter<true, false>, smp)) return rc;
    {
      PF_KERNEL("k_fscatter_build", st);
      k_fscatter<false, false><<<nch_b, FT, smb, st>>>((const long long*)build_key, build_group,
                                                       nullptr, 0, n_build, chunk_b, logB, B,
                                                       l.hist_b, l.start, l.pkey, l.pgrp);
    }
    {
      PF_KERNEL("k_fscatter_probe", st);
      k_fscatter<true, false><<<nch_p, FT, smp, st>>>((const long long*)probe_fk, probe_price,
                                                      (const long long*)probe_disc, scale, n_probe,
                                                      chunk_p, logB, B, l.hist_p, l.start + B,
                                                      l.pfk, l.pval);
    }
  }
  return ok();
}

// Both sides' bucket counts and starts (the counted first pass and the round
// path): per-chunk histograms, per-bucket chunk offsets, the starts, and the
// counts copied into `hc` (pinned) behind the returned event.
int count_buckets(const int64_t* build_key, long long n_build, const int64_t* probe_fk,
                  long long n_probe, int logB, int B, const JaLayout& l, long long* hc,
                  cudaEvent_t* ev, cudaStream_t st) {
  long long chunk_b, chunk_p;
  int nch_b, nch_p;
  chunking(n_build, &chunk_b, &nch_b);
  chunking(n_probe, &chunk_p, &nch_p);
  const size_t hsm = (size_t)B * sizeof(int);
  if (int rc = opt_in_smem((const void*)k_fhist, hsm)) return rc;
  {
    PF_KERNEL("k_fhist", st);
    k_fhist<<<nch_b, FT, hsm, st>>>((const long long*)build_key, n_build, chunk_b, logB, B, l.hist_b);
  }
  {
    PF_KERNEL("k_fhist", st);
    k_fhist<<<nch_p, FT, hsm, st>>>((const long long*)probe_fk, n_probe, chunk_p, logB, B, l.hist_p);
  }
  PF_LAUNCH("k_fhist");
  {
    PF_KERNEL("k_fscan", st);
    k_fscan<<<(B + 31) / 32, FT, 0, st>>>(l.hist_b, nch_b, B, l.cnt);
  }
  {
    PF_KERNEL("k_fscan", st);
    k_fscan<<<(B + 31) / 32, FT, 0, st>>>(l.hist_p, nch_p, B, l.cnt + B);
  }
  PF_LAUNCH("k_fscan");
  PF_CUDA(cudaMemcpyAsync(l.start, l.cnt, 2 * B * sizeof(long long), cudaMemcpyDeviceToDevice, st));
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.start, B, l.total, nullptr);
  }
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.start + B, B, l.total + 1, nullptr);
  }
  PF_LAUNCH("k_scan_counts");
  PF_CUDA(cudaMemcpyAsync(hc, l.cnt, 2 * B * sizeof(long long), cudaMemcpyDeviceToHost, st));
  return record_event(st, ev);
}

// Launch shape of a tile scatter: opt in to its shared memory, then one
// block a tile up to the resident blocks of every SM.
template <int MODE, bool AOS, int BINS, int RI>
int p2_launch(const P2Args& a, long long ntiles, size_t extra_smem, const char* name,
              cudaStream_t st) {
  if (ntiles <= 0) return ok();
  const size_t sm = sizeof(P2Smem<BINS, P2T * RI>) + extra_smem;
  // records leave shared memory by bulk copies (the workspace starts on a
  // 256-byte boundary, so every record output is 16-byte aligned), columns by
  // thread stores
  auto kern = k_p2_scatter<MODE, AOS, BINS, RI, AOS>;
  if (int rc = opt_in_smem((const void*)kern, sm)) return rc;
  int per_sm = 0;
  PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P2T, sm));
  const unsigned g = (unsigned)std::max<long long>(
      1, std::min<long long>(ntiles, (long long)std::max(1, per_sm) * sm_count()));
  {
    PF_KERNEL(name, st);
    kern<<<g, P2T, sm, st>>>(a);
  }
  PF_LAUNCH(name);
  return ok();
}

// The shared-memory path's first pass: both sides hashed and scattered by
// the tile scatter into B buckets, from the cursors in l.cur1; cap > 0: into
// regions of cap rows a bucket (an overflow raises ovf[0]).
int first_pass(const int64_t* build_key, const int32_t* build_group, long long n_build,
               const int64_t* probe_fk, const int64_t* probe_price, const int64_t* probe_disc,
               long long scale, long long n_probe, int logB, int B, const long long cap[2],
               const JaLayout& l, cudaStream_t st) {
  P2Args b{};
  b.key = (const long long*)build_key;
  b.val = build_group;
  b.n = n_build;
  b.logS = b.logB2 = logB;
  b.cursor = l.cur1;
  b.cap = cap[0];
  b.ovf = l.ovf;
  b.key_out = l.pkey;
  b.val_out = l.pgrp;
  P2Args p{};
  p.key = (const long long*)probe_fk;
  p.val = probe_price;
  p.disc = (const long long*)probe_disc;
  p.scale = scale;
  p.n = n_probe;
  p.logS = p.logB2 = logB;
  p.cursor = l.cur1 + B;
  p.cap = cap[1];
  p.ovf = l.ovf;
  p.rec_out = l.prec;
  constexpr int tb = P2TILE, tp = P2T * P2RI2;
  const long long nbt = (n_build + tb - 1) / tb, npt = (n_probe + tp - 1) / tp;
  if (B <= P2BINS) {
    if (int rc = p2_launch<1, false, P2BINS, P2I>(b, nbt, 0, "k_fscatter_build", st)) return rc;
    return p2_launch<2, true, P2BINS, P2RI2>(p, npt, 0, "k_fscatter_probe", st);
  }
  if (int rc = p2_launch<1, false, P1BINS, P2I>(b, nbt, 0, "k_fscatter_build", st)) return rc;
  return p2_launch<2, true, P1BINS, P2RI2>(p, npt, 0, "k_fscatter_probe", st);
}

// The second pass of one side into sub-partitions.  counted: per-segment
// histograms and a scan give every sub-partition's exact start (rows
// contiguous; beg = start2, end = start2 + 1); else regions of cap2 rows
// (beg = their starts, end = the cursors after the scatter; an overflow
// raises ovf[1]).
// The first pass's output as the second pass reads it: build rows as (hash,
// group) columns, probe rows as records, partition p of a side at the rows
// the device array `part` gives (starts of both sides, then rows).
struct P1View {
  const long long* bkey;
  const int* bgrp;
  const P2Row* prec;
};

int second_pass(const JaLayout& l, const P1View& v, int side, bool counted, long long cap2,
                int B, int logB2, int logS, const long long* hcnt, const long long* d_pstart,
                const long long* d_pcnt, const unsigned long long** beg,
                const unsigned long long** end, cudaStream_t st) {
  const long long S = (long long)B << logB2;
  unsigned long long* cur = l.cur2 + side * l.s_max;
  unsigned long long* start = l.start2 + side * (l.s_max + 1);
  const int sms = sm_count();
  if (counted) {
    std::vector<int2> seg;
    std::vector<int> pseg((size_t)B + 1);
    for (int p = 0; p < B; ++p) {
      pseg[p] = (int)seg.size();
      for (long long j = 0; j * P2SEG < hcnt[p]; ++j) seg.push_back(make_int2(p, (int)j));
    }
    pseg[B] = (int)seg.size();
    if ((long long)seg.size() > l.nseg_max[side])
      return fail(PF_ENOSPACE, "join_aggregate: %zu pass-2 segments, room for %lld",
                  seg.size(), l.nseg_max[side]);
    // pageable sources: the copies take the data before they return
    if (!seg.empty())
      PF_CUDA(cudaMemcpyAsync(l.seg2[side], seg.data(), seg.size() * sizeof(int2),
                              cudaMemcpyHostToDevice, st));
    PF_CUDA(cudaMemcpyAsync(l.pseg2[side], pseg.data(), pseg.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
    SegArgs g{l.seg2[side], (int)seg.size(), d_pstart, d_pcnt, logS, logB2};
    if (g.nseg) {
      PF_KERNEL("k_p2_hist", st);
      const unsigned grid = (unsigned)std::min<long long>(g.nseg, sms * 4LL);
      if (side) k_p2_hist<true><<<grid, P2T, 0, st>>>(nullptr, v.prec, g, l.hist2[side]);
      else k_p2_hist<false><<<grid, P2T, 0, st>>>(v.bkey, nullptr, g, l.hist2[side]);
    }
    PF_LAUNCH("k_p2_hist");
    {
      PF_KERNEL("k_p2_colsum", st);
      k_p2_colsum<<<(unsigned)((S + 255) / 256), 256, 0, st>>>(
          l.hist2[side], l.pseg2[side], (int)S, logB2, l.tot2 + side * l.s_max);
    }
    PF_LAUNCH("k_p2_colsum");
    if (int rc = scan_i64(l.tot2 + side * l.s_max, (long long*)start, S, false,
                          (long long*)start + S, l.scan2, st))
      return rc;
    PF_CUDA(cudaMemcpyAsync(cur, start, S * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                            st));
    *beg = start;
    *end = start + 1;
  } else {
    {
      PF_KERNEL("k_region_starts", st);
      k_region_starts<<<(unsigned)std::min<long long>((S + 255) / 256, sms * 8LL), 256, 0, st>>>(
          cur, l.beg2 + side * l.s_max, S, cap2);
    }
    PF_LAUNCH("k_region_starts");
    *beg = l.beg2 + side * l.s_max;
    *end = cur;
  }
  // tiles partition by partition (hcnt null: already planned on the device,
  // their number known there only)
  const long long tile = side ? (long long)P2T * P2I_AOS : (long long)P2TILE;
  long long nt = LLONG_MAX;
  if (hcnt) {
    std::vector<int> ts((size_t)B + 1);
    nt = 0;
    for (int p = 0; p < B; ++p) {
      ts[p] = (int)nt;
      nt += (hcnt[p] + tile - 1) / tile;
    }
    ts[B] = (int)nt;
    if (nt >= INT_MAX) return fail(PF_EINVAL, "join_aggregate: too many second-pass tiles");
    PF_CUDA(cudaMemcpyAsync(l.tstart[side], ts.data(), ts.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  }
  P2Args a{};
  a.pstart = d_pstart;
  a.pcnt = d_pcnt;
  a.tstart = l.tstart[side];
  a.B = B;
  a.logS = logS;
  a.logB2 = logB2;
  a.cursor = cur;
  a.cap = counted ? 0 : cap2;
  a.ovf = l.ovf + 1;
  a.skip = hcnt ? nullptr : l.ovf;
  const size_t extra = ((size_t)B + 1) * sizeof(int);
  if (side) {
    a.rec = v.prec;
    a.rec_out = l.prec2;
    return p2_launch<0, true, P2BINS, P2I_AOS>(a, nt, extra, "k_p2_scatter", st);
  }
  a.key = v.bkey;
  a.val = v.bgrp;
  a.key_out = l.pkey2;
  a.val_out = l.pgrp2;
  return p2_launch<0, false, P2BINS, P2I>(a, nt, extra, "k_p2_scatter", st);
}

// The shared-memory path after the first pass: the second radix pass of B
// partitions (part: starts of both sides, then rows, on the host; logB the
// bits of the hash the partitions share) into sub-partitions of about
// kn.target build rows, the join per sub-partition into the slab (zeroed by
// the caller), the slab split.  A side whose regions would not fit its
// buffer, or every side after an overflow, takes the counted second pass.
// Keys are mix64 hashes here.
//
// dev (the first pass into regions, its plan made on the device by
// k_pass1_plan; part unused): partitions are taken at their regions' size,
// the regions the workspace was sized for, and the host waits once, at the
// end, for both passes' overflow words; *redo is then 1 when the first pass
// overflowed (nothing was joined: run everything counted), 2 when only the
// second did (run the second pass counted from the first pass's cursors).
int join_smem(const JaLayout& l, const P1View& v, const Knobs& kn, int B, int logB,
              const std::vector<long long>& part, long long group_min, long long n_groups,
              int64_t* sum_out, int64_t* count_out, int64_t* stats_out, long long* hstage,
              cudaStream_t st, bool dev = false, int* redo = nullptr) {
  const long long* hc = nullptr;
  long long maxp[2] = {0, 0};
  if (dev) {
    maxp[0] = l.cap1[0];
    maxp[1] = l.cap1[1];
  } else {
    // pageable source: the copy takes the data before it returns
    PF_CUDA(cudaMemcpyAsync(l.pstart, part.data(), 4 * (size_t)B * sizeof(long long),
                            cudaMemcpyHostToDevice, st));
    hc = part.data() + 2 * (size_t)B;
    for (int side = 0; side < 2; ++side)
      for (int p = 0; p < B; ++p) maxp[side] = std::max(maxp[side], hc[(size_t)side * B + p]);
  }
  int logB2 = 0;
  while ((maxp[0] >> logB2) > kn.target && logB2 < P2MAXLOG &&
         ((long long)B << (logB2 + 1)) <= l.s_max)
    ++logB2;
  const int logS = logB + logB2;
  // sub-partitions: each of the B partitions split 2^logB2 ways (B need
  // not be 2^logB: a rank of a sharded join holds some of the buckets)
  const long long S = (long long)B << logB2;
  const int sms = sm_count();
  bool counted[2];
  long long cap2[2];
  for (int side = 0; side < 2; ++side) {
    cap2[side] = region_rows((double)maxp[side] / (double)(1LL << logB2), region_var(side));
    counted[side] = kn.counted || S * cap2[side] > l.rows2[side];
  }
  if (dev && (counted[0] || counted[1])) {
    // the workspace was sized for these regions, so this does not happen:
    // if it did, the host's plan takes over (after the first pass's word)
    PF_CUDA(cudaMemcpyAsync(hstage, l.ovf, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st));
    if (int rc = wait_stream(st)) return rc;
    *redo = hstage[0] ? 1 : 2;
    return ok();
  }
  for (int attempt = 0; attempt < 2; ++attempt) {
    PF_CUDA(cudaMemsetAsync(l.ovf + 1, 0, sizeof(unsigned long long), st));
    const unsigned long long *bbeg, *bend, *pbeg, *pend;
    if (int rc = second_pass(l, v, 0, counted[0], cap2[0], B, logB2, logS, hc, l.pstart,
                             l.pstart + 2 * B, &bbeg, &bend, st))
      return rc;
    if (int rc = second_pass(l, v, 1, counted[1], cap2[1], B, logB2, logS, hc ? hc + B : nullptr,
                             l.pstart + B, l.pstart + 3 * B, &pbeg, &pend, st))
      return rc;
    SJArgs a{};
    a.bkey = l.pkey2;
    a.bgrp = l.pgrp2;
    a.prec = l.prec2;
    a.bbeg = bbeg;
    a.bend = bend;
    a.pbeg = pbeg;
    a.pend = pend;
    a.S = S;
    a.logS = logS;
    a.group_min = group_min;
    a.n_groups = n_groups;
    a.slab = l.slab;
    a.stats = (unsigned long long*)stats_out;
    a.counter = l.sj_counter;
    a.ovf = l.ovf + 1;
    a.ovf1 = dev ? l.ovf : nullptr;
    PF_CUDA(cudaMemsetAsync(l.sj_counter, 0, sizeof(unsigned long long), st));
    if (kn.table) {
      const size_t smem = sizeof(SJFSmem);
      if (int rc = opt_in_smem((const void*)k_sjoin_fp, smem)) return rc;
      int per_sm = 0;
      PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sjoin_fp, SJF_T, smem));
      PF_KERNEL("k_sjoin", st);
      k_sjoin_fp<<<std::max(1, per_sm) * sms, SJF_T, smem, st>>>(a);
    } else {
      const size_t smem = sizeof(SJSmem);
      if (int rc = opt_in_smem((const void*)k_sjoin, smem)) return rc;
      int per_sm = 0;
      PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sjoin, SJT, smem));
      PF_KERNEL("k_sjoin", st);
      k_sjoin<<<std::max(1, per_sm) * sms, SJT, smem, st>>>(a);
    }
    PF_LAUNCH("k_sjoin");
    {
      PF_KERNEL("k_split", st);
      k_split<<<(unsigned)std::max<long long>(
                    1, std::min<long long>((n_groups + 255) / 256, sms * 8LL)),
                256, 0, st>>>(l.slab, n_groups, (long long*)sum_out, (long long*)count_out);
    }
    PF_LAUNCH("k_split");
    g_counted_passes = (g_counted_passes & 1) | (counted[0] || counted[1] ? 2 : 0);
    if (counted[0] && counted[1]) return ok();
    // regions: whether one overflowed (then nothing was joined)
    if (dev) {
      PF_CUDA(cudaMemcpyAsync(hstage, l.ovf, 2 * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, st));
      if (int rc = wait_stream(st)) return rc;
      *redo = hstage[0] ? 1 : hstage[1] ? 2 : 0;
      return ok();
    }
    PF_CUDA(cudaMemcpyAsync(hstage, l.ovf + 1, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    if (int rc = wait_stream(st)) return rc;
    if (!hstage[0]) return ok();
    counted[0] = counted[1] = true;
  }
  return fail(PF_ECUDA, "join_aggregate: the counted second pass overflowed");
}
}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int pf_join_aggregate_pick_b(int64_t n_build, int64_t n_probe) {
  (void)n_probe;
  const long long target = std::max<long long>(1, round_rows() / 2);
  long long b = 1;
  while (b < FB_MAX && n_build / b > target) b <<= 1;
  return (int)b;
}

extern "C" int pf_join_aggregate_counted_passes(void) { return g_counted_passes; }

extern "C" size_t pf_join_aggregate_workspace_ex(int64_t n_build, int64_t n_probe, int B,
                                                 int64_t n_groups, const pf_join_knobs* knobs) {
  if (B < 1) B = 1;
  Arena a(nullptr, 0);
  ja_layout(a, n_build, n_probe, B, n_groups, resolve_knobs(knobs));
  return a.used + 256;
}

extern "C" size_t pf_join_aggregate_workspace(int64_t n_build, int64_t n_probe, int B,
                                              int64_t n_groups) {
  return pf_join_aggregate_workspace_ex(n_build, n_probe, B, n_groups, nullptr);
}

extern "C" int pf_join_aggregate(const int64_t* build_key, const int32_t* build_group,
                                 int64_t n_build, const int64_t* probe_fk,
                                 const int64_t* probe_price, const int64_t* probe_disc,
                                 int64_t scale, int64_t n_probe, int B, int64_t group_min,
                                 int64_t n_groups, int64_t* sum_out, int64_t* count_out,
                                 int64_t* stats_out, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  return pf_join_aggregate_ex(build_key, build_group, n_build, probe_fk, probe_price, probe_disc,
                              scale, n_probe, B, group_min, n_groups, sum_out, count_out,
                              stats_out, nullptr, workspace, workspace_bytes, stream);
}

extern "C" int pf_join_aggregate_ex(const int64_t* build_key, const int32_t* build_group,
                                    int64_t n_build, const int64_t* probe_fk,
                                    const int64_t* probe_price, const int64_t* probe_disc,
                                    int64_t scale, int64_t n_probe, int B, int64_t group_min,
                                    int64_t n_groups, int64_t* sum_out, int64_t* count_out,
                                    int64_t* stats_out, const pf_join_knobs* knobs,
                                    void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const Knobs kn = resolve_knobs(knobs);
  if (knobs && (knobs->path < 0 || knobs->path > 1 || knobs->sub_rows < 0))
    return fail(PF_EINVAL, "join_aggregate: knobs path %d, sub_rows %d", knobs->path,
                knobs->sub_rows);
  if (B < 1 || B > FB_MAX || (B & (B - 1)))
    return fail(PF_EINVAL, "join_aggregate: B must be a power of two in [1, %d], got %d", FB_MAX, B);
  if (n_build < 0 || n_probe < 0 || n_groups < 1 || n_groups > 0xfffffffeLL)
    return fail(PF_EINVAL, "join_aggregate: bad sizes (build %lld, probe %lld, groups %lld)",
                (long long)n_build, (long long)n_probe, (long long)n_groups);
  if (n_build >= (1LL << 40) || n_probe >= (1LL << 40))
    return fail(PF_EINVAL, "join_aggregate: at most 2^40 rows a side");
  Arena ar(workspace, workspace_bytes);
  JaLayout l = ja_layout(ar, n_build, n_probe, B, n_groups, kn);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "join_aggregate: workspace of %zu bytes, %zu needed",
                workspace_bytes, ar.used);
  const int logB = log2_exact((uint64_t)B);
  PF_CUDA(cudaMemsetAsync(stats_out, 0, 4 * sizeof(long long), st));
  if (n_build == 0 || n_probe == 0) {
    PF_CUDA(cudaMemsetAsync(sum_out, 0, n_groups * sizeof(long long), st));
    PF_CUDA(cudaMemsetAsync(count_out, 0, n_groups * sizeof(long long), st));
    return ok();
  }
  PF_CUDA(cudaMemsetAsync(l.slab, 0, 2 * n_groups * sizeof(unsigned long long), st));

  long long* hc = pinned_counts(2 * (size_t)B + 8);
  if (!hc) return fail(PF_ECUDA, "join_aggregate: no pinned staging buffer");
  const int sms = sm_count();
  if (kn.smem) {
    // 1: the first pass into regions of cap1 rows a bucket, from their starts
    bool counted = kn.counted != 0;
    std::vector<long long> part(4 * (size_t)B);  // starts, then rows, of both sides
    if (!counted) {
      for (int side = 0; side < 2; ++side) {
        PF_KERNEL("k_region_starts", st);
        k_region_starts<<<(unsigned)std::max(1, (B + 255) / 256), 256, 0, st>>>(
            l.cur1 + (size_t)side * B, nullptr, B, l.cap1[side]);
      }
      PF_LAUNCH("k_region_starts");
      PF_CUDA(cudaMemsetAsync(l.ovf, 0, sizeof(unsigned long long), st));
      if (int rc = first_pass(build_key, build_group, n_build, probe_fk, probe_price, probe_disc,
                              scale, n_probe, logB, B, l.cap1, l, st))
        return rc;
      // the second pass and the join queued behind it, planned on the
      // device from the cursors (the buckets' ends); one host wait, at the end
      {
        PF_KERNEL("k_pass1_plan", st);
        k_pass1_plan<<<1, 1024, 0, st>>>(l.cur1, B, l.cap1[0], l.cap1[1], P2TILE,
                                         (long long)P2T * P2I_AOS, l.pstart, l.tstart[0],
                                         l.tstart[1]);
      }
      PF_LAUNCH("k_pass1_plan");
      g_counted_passes = 0;
      int redo = 0;
      if (int rc = join_smem(l, P1View{l.pkey, l.pgrp, l.prec}, kn, B, logB, part, group_min,
                             n_groups, sum_out, count_out, stats_out, hc, st, true, &redo))
        return rc;
      if (redo == 0) return ok();
      if (redo == 1) {
        counted = true;  // the first pass overflowed: nothing was joined
      } else {
        // the second pass overflowed: again from the first pass's cursors,
        // the second pass counted
        PF_CUDA(cudaMemcpyAsync(hc, l.cur1, 2 * B * sizeof(long long), cudaMemcpyDeviceToHost,
                                st));
        if (int rc = wait_stream(st)) return rc;
        for (int side = 0; side < 2; ++side)
          for (int p = 0; p < B; ++p) {
            const size_t i = (size_t)side * B + p;
            part[i] = p * l.cap1[side];
            part[2 * (size_t)B + i] = hc[i] - part[i];
          }
        Knobs kc = kn;
        kc.counted = 1;
        return join_smem(l, P1View{l.pkey, l.pgrp, l.prec}, kc, B, logB, part, group_min,
                         n_groups, sum_out, count_out, stats_out, hc, st);
      }
    }
    if (counted) {
      // a bucket overflowed its region (or counting was asked for): count
      // first, then scatter from the exact starts
      const long long none[2] = {0, 0};
      cudaEvent_t ev;
      if (int rc = count_buckets(build_key, n_build, probe_fk, n_probe, logB, B, l, hc, &ev, st))
        return rc;
      PF_CUDA(cudaMemcpyAsync(l.cur1, l.start, 2 * B * sizeof(long long),
                              cudaMemcpyDeviceToDevice, st));
      if (int rc = first_pass(build_key, build_group, n_build, probe_fk, probe_price, probe_disc,
                              scale, n_probe, logB, B, none, l, st))
        return rc;
      if (int rc = wait_event(ev)) return rc;
      for (int side = 0; side < 2; ++side) {
        long long run = 0;
        for (int p = 0; p < B; ++p) {
          const size_t i = (size_t)side * B + p;
          part[i] = run;
          part[2 * (size_t)B + i] = hc[i];
          run += hc[i];
        }
      }
    }
    g_counted_passes = counted ? 1 : 0;
    return join_smem(l, P1View{l.pkey, l.pgrp, l.prec}, kn, B, logB, part, group_min, n_groups,
                     sum_out, count_out, stats_out, hc, st);
  }

  // the round path: counts, then the first pass, queued while the host waits
  // for the counts
  g_counted_passes = 1;
  cudaEvent_t ev;
  if (int rc = count_buckets(build_key, n_build, probe_fk, n_probe, logB, B, l, hc, &ev, st))
    return rc;
  long long chunk_b, chunk_p;
  int nch_b, nch_p;
  chunking(n_build, &chunk_b, &nch_b);
  chunking(n_probe, &chunk_p, &nch_p);
  const bool tma = aligned16(build_key) && aligned16(build_group) && aligned16(probe_fk) &&
                   aligned16(probe_price) && (!probe_disc || aligned16(probe_disc)) &&
                   getenv("PF_NO_TMA") == nullptr;
  if (int rc = fscatter_rounds(tma, build_key, build_group, n_build, probe_fk, probe_price,
                               probe_disc, scale, n_probe, chunk_b, nch_b, chunk_p, nch_p, logB,
                               B, l, stats_out, st))
    return rc;
  PF_LAUNCH("k_fscatter");
  if (int rc = wait_event(ev)) return rc;

  // 4: plan the rounds from the counts
  const long long cap_rows = l.table_slots / 2;
  std::vector<Round> rounds;
  long long bs = 0, ps = 0;
  for (int p = 0; p < B;) {
    const long long nbp = hc[p], npp = hc[B + p];
    if (nbp > cap_rows) {
      // one partition over the budget: slices of its build rows
      for (long long s0 = 0; s0 < nbp; s0 += cap_rows) {
        const long long s1 = std::min(nbp, s0 + cap_rows);
        rounds.push_back(Round{p, p + 1, bs + s0, bs + s1, ps, ps + npp, 2 * (s1 - s0)});
      }
      bs += nbp;
      ps += npp;
      ++p;
      continue;
    }
    Round r{p, p, bs, bs, ps, ps, 0};
    long long rows = 0;
    while (p < B && hc[p] <= cap_rows && rows + hc[p] <= cap_rows) {
      rows += hc[p];
      bs += hc[p];
      ps += hc[B + p];
      ++p;
    }
    r.p1 = p;
    r.b_hi = bs;
    r.p_hi = ps;
    rounds.push_back(r);
  }
  {
    PF_KERNEL("k_plan", st);
    k_plan<<<1, 32, 0, st>>>(l.cnt, B, cap_rows, l.reg);
  }
  PF_LAUNCH("k_plan");
  PF_CUDA(cudaMemsetAsync(l.table, 0, 2 * l.table_slots * sizeof(Slot), st));
  if ((long long)rounds.size() + 1 > l.max_launches)
    return fail(PF_EINVAL, "join_aggregate: %zu rounds exceed the planned %lld", rounds.size(),
                l.max_launches - 1);
  PF_CUDA(cudaMemsetAsync(l.counters, 0, (rounds.size() + 1) * sizeof(unsigned), st));

  RoundArgs a{};
  a.bkey = l.pkey;
  a.bgrp = l.pgrp;
  a.pfk = l.pfk;
  a.pval = l.pval;
  a.reg_off = l.reg;
  a.reg_cap = l.reg + B;
  a.logB = logB;
  a.group_min = group_min;
  a.n_groups = n_groups;
  a.slab = l.slab;
  a.stats = (unsigned long long*)stats_out;
  auto round_args = [&](long long r) {
    RoundArgs x = a;
    if (r < 0 || r >= (long long)rounds.size()) {
      x.b_lo = x.b_hi = x.p_lo = x.p_hi = 0;
      x.p0 = x.p1 = 0;
      x.slice_cap = 0;
      x.table = l.table;
      x.tag = 0;
      return x;
    }
    const Round& R = rounds[r];
    x.b_lo = R.b_lo;
    x.b_hi = R.b_hi;
    x.p_lo = R.p_lo;
    x.p_hi = R.p_hi;
    x.slice_cap = R.slice_cap;
    x.p0 = R.p0;
    x.p1 = R.p1;
    x.tag = (unsigned)(r + 1);
    x.table = l.table + (r & 1) * l.table_slots;
    return x;
  };
  // launch k: probe round k - 1 and build round k
  for (long long k = 0; k <= (long long)rounds.size(); ++k) {
    RoundArgs pa = round_args(k - 1), ba = round_args(k);
    if (pa.b_hi == pa.b_lo) pa.p_hi = pa.p_lo;  // no build rows: nothing to match
    const long long np_rows = pa.p_hi - pa.p_lo, nb_rows = ba.b_hi - ba.b_lo;
    const int units_p = (int)((np_rows + UROWS - 1) / UROWS);
    const int units_b = (int)((nb_rows + UROWS - 1) / UROWS);
    if (units_p + units_b == 0) continue;
    const int nregp = np_rows > 0 ? (pa.slice_cap > 0 ? 1 : pa.p1 - pa.p0) : 0;
    const int nregb = nb_rows > 0 ? (ba.slice_cap > 0 ? 1 : ba.p1 - ba.p0) : 0;
    const size_t rsm = sizeof(ProbeStage) + (size_t)std::max(1, nregp + nregb) * sizeof(uint2);
    if (int rc = opt_in_smem((const void*)k_fround, rsm)) return rc;
    const unsigned g = (unsigned)std::max<long long>(
        1, std::min<long long>(units_p + units_b, (long long)sms * PF_PROBE_GRID));
    {
      PF_KERNEL("k_fround", st);
      k_fround<<<g, PT2, rsm, st>>>(pa, ba, l.counters + k, units_p, units_b);
    }
  }
  PF_LAUNCH("k_fround");
  {
    PF_KERNEL("k_split", st);
    k_split<<<(unsigned)std::max<long long>(1, std::min<long long>((n_groups + 255) / 256, sms * 8LL)),
              256, 0, st>>>(l.slab, n_groups, (long long*)sum_out, (long long*)count_out);
  }
  PF_LAUNCH("k_split");
  return ok();
}

namespace {
struct GfLayout {
  long long* bcnt;
  long long* total;
};
GfLayout gf_layout(Arena& a, int64_t n) {
  GfLayout l{};
  l.bcnt = a.take<long long>((n + CB - 1) / CB + 1);
  l.total = a.take<long long>(1);
  return l;
}
}  // namespace

extern "C" size_t pf_groups_finish_workspace(int64_t n_groups) {
  Arena a(nullptr, 0);
  gf_layout(a, n_groups);
  return a.used + 256;
}

extern "C" int pf_groups_finish(const int64_t* sum, const int64_t* count, int64_t group_min,
                                int64_t n_groups, int64_t* keys_out, int64_t* sums_out,
                                int64_t* counts_out, int64_t* host_out, void* workspace,
                                size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  Arena ar(workspace, workspace_bytes);
  GfLayout l = gf_layout(ar, n_groups);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "groups_finish: workspace of %zu bytes, %zu needed", workspace_bytes,
                ar.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  if (n_groups <= 0) {
    host_out[0] = 0;
    return ok();
  }
  const unsigned nblk = blocks_for(n_groups, CB);
  {
    PF_KERNEL("k_gcount", st);
    k_gcount<<<nblk, CT, 0, st>>>((const long long*)count, n_groups, l.bcnt);
  }
  PF_LAUNCH("k_gcount");
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.bcnt, nblk, l.total, host_dev);
  }
  PF_LAUNCH("k_scan_counts");
  cudaEvent_t ev;
  if (int rc = record_event(st, &ev)) return rc;
  {
    PF_KERNEL("k_gemit", st);
    k_gemit<<<nblk, CT, 0, st>>>((const long long*)sum, (const long long*)count, n_groups,
                                 group_min, l.bcnt, (long long*)keys_out, (long long*)sums_out,
                                 (long long*)counts_out);
  }
  PF_LAUNCH("k_gemit");
  if (int rc = wait_event(ev)) return rc;
  return ok();
}

// ---- the join sharded over ranks: its two local phases ----------------------------
//
// Rank-local halves of pf_join_aggregate for a join whose rows are spread
// over ranks: pf_join_partition hashes and radix-partitions a rank's rows
// (counted, so every bucket is contiguous and the buckets can be sent to
// their owners as they lie); after the exchange, pf_join_aggregate_buckets
// runs the second radix pass and the join over the buckets a rank owns,
// each bucket's rows contiguous, into a dense slab the ranks then add up.

namespace pf {
namespace {
JaLayout partition_layout(Arena& a, long long nb, long long np, int B) {
  JaLayout l{};
  long long chunk;
  int nb_ch, np_ch;
  chunking(nb, &chunk, &nb_ch);
  chunking(np, &chunk, &np_ch);
  l.hist_b = a.take<int>((size_t)nb_ch * B);
  l.hist_p = a.take<int>((size_t)np_ch * B);
  l.cnt = a.take<long long>(2 * (size_t)B);
  l.start = a.take<long long>(2 * (size_t)B);
  l.total = a.take<long long>(2);
  l.cur1 = a.take<unsigned long long>(2 * (size_t)B);
  l.ovf = a.take<unsigned long long>(2);
  return l;
}

JaLayout buckets_layout(Arena& a, const int64_t* counts, int nbk, long long n_groups,
                        const Knobs& kn) {
  JaLayout l{};
  long long rows[2] = {0, 0}, maxp[2] = {0, 0};
  for (int side = 0; side < 2; ++side)
    for (int p = 0; p < nbk; ++p) {
      rows[side] += counts[(size_t)side * nbk + p];
      maxp[side] = std::max<long long>(maxp[side], counts[(size_t)side * nbk + p]);
    }
  l.slab = a.take<unsigned long long>(2 * (size_t)std::max<long long>(n_groups, 1));
  l.ovf = a.take<unsigned long long>(2);
  take_second_pass(a, l, rows[0], rows[1], nbk, maxp, kn.target);
  return l;
}
}  // namespace
}  // namespace pf

extern "C" size_t pf_join_partition_workspace(int64_t n_build, int64_t n_probe, int B) {
  if (B < 1) B = 1;
  Arena a(nullptr, 0);
  partition_layout(a, n_build, n_probe, B);
  return a.used + 256;
}

extern "C" int pf_join_partition(const int64_t* build_key, const int32_t* build_group,
                                 int64_t n_build, const int64_t* probe_fk,
                                 const int64_t* probe_price, const int64_t* probe_disc,
                                 int64_t scale, int64_t n_probe, int B, int64_t* build_hash_out,
                                 int32_t* build_group_out, int64_t* probe_rec_out,
                                 int64_t* host_counts, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (B < 1 || B > FB_MAX || (B & (B - 1)))
    return fail(PF_EINVAL, "join_partition: B must be a power of two in [1, %d], got %d", FB_MAX,
                B);
  if (n_build < 0 || n_probe < 0 || n_build >= (1LL << 40) || n_probe >= (1LL << 40))
    return fail(PF_EINVAL, "join_partition: bad sizes (build %lld, probe %lld)",
                (long long)n_build, (long long)n_probe);
  if (!host_counts) return fail(PF_EINVAL, "join_partition: null host_counts");
  Arena ar(workspace, workspace_bytes);
  JaLayout l = partition_layout(ar, n_build, n_probe, B);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "join_partition: workspace of %zu bytes, %zu needed",
                workspace_bytes, ar.used);
  if (n_build == 0 && n_probe == 0) {
    for (int i = 0; i < 2 * B; ++i) host_counts[i] = 0;
    return ok();
  }
  l.pkey = (long long*)build_hash_out;
  l.pgrp = build_group_out;
  l.prec = (P2Row*)probe_rec_out;
  const int logB = log2_exact((uint64_t)B);
  cudaEvent_t ev;
  if (int rc = count_buckets(build_key, n_build, probe_fk, n_probe, logB, B, l,
                             (long long*)host_counts, &ev,
                             st))
    return rc;
  PF_CUDA(cudaMemcpyAsync(l.cur1, l.start, 2 * B * sizeof(long long), cudaMemcpyDeviceToDevice,
                          st));
  const long long none[2] = {0, 0};
  if (int rc = first_pass(build_key, build_group, n_build, probe_fk, probe_price, probe_disc,
                          scale, n_probe, logB, B, none, l, st))
    return rc;
  return wait_event(ev);
}

extern "C" size_t pf_join_aggregate_buckets_workspace(const int64_t* counts, int nbk,
                                                      int64_t n_groups,
                                                      const pf_join_knobs* knobs) {
  if (!counts || nbk < 1) return 256;
  Arena a(nullptr, 0);
  buckets_layout(a, counts, nbk, n_groups, resolve_knobs(knobs));
  return a.used + 256;
}

extern "C" int pf_join_aggregate_buckets(const int64_t* build_hash, const int32_t* build_group,
                                         const int64_t* probe_rec, const int64_t* counts,
                                         int nbk, int logB, int64_t group_min, int64_t n_groups,
                                         int64_t* sum_out, int64_t* count_out,
                                         int64_t* stats_out, const pf_join_knobs* knobs,
                                         void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const Knobs kn = resolve_knobs(knobs);
  if (!kn.smem) return fail(PF_EINVAL, "join_aggregate_buckets: the shared-memory join only");
  if (!counts || nbk < 1 || logB < 0 || logB > 12 || nbk > (1 << logB))
    return fail(PF_EINVAL, "join_aggregate_buckets: %d buckets of %d hash bits", nbk, logB);
  if (n_groups < 1 || n_groups > 0xfffffffeLL)
    return fail(PF_EINVAL, "join_aggregate_buckets: bad group count %lld", (long long)n_groups);
  Arena ar(workspace, workspace_bytes);
  JaLayout l = buckets_layout(ar, counts, nbk, n_groups, kn);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "join_aggregate_buckets: workspace of %zu bytes, %zu needed",
                workspace_bytes, ar.used);
  PF_CUDA(cudaMemsetAsync(stats_out, 0, 4 * sizeof(long long), st));
  std::vector<long long> part(4 * (size_t)nbk);
  long long tot[2] = {0, 0};
  for (int side = 0; side < 2; ++side)
    for (int p = 0; p < nbk; ++p) {
      const size_t i = (size_t)side * nbk + p;
      if (counts[i] < 0) return fail(PF_EINVAL, "join_aggregate_buckets: negative count");
      part[i] = tot[side];
      part[2 * (size_t)nbk + i] = counts[i];
      tot[side] += counts[i];
    }
  if (tot[0] == 0 || tot[1] == 0) {
    PF_CUDA(cudaMemsetAsync(sum_out, 0, n_groups * sizeof(long long), st));
    PF_CUDA(cudaMemsetAsync(count_out, 0, n_groups * sizeof(long long), st));
    return ok();
  }
  PF_CUDA(cudaMemsetAsync(l.slab, 0, 2 * n_groups * sizeof(unsigned long long), st));
  long long* hc = pinned_counts(8);
  if (!hc) return fail(PF_ECUDA, "join_aggregate_buckets: no pinned staging buffer");
  return join_smem(l, P1View{(const long long*)build_hash, build_group, (const P2Row*)probe_rec},
                   kn, nbk, logB, part, group_min, n_groups, sum_out, count_out, stats_out, hc,
                   st);
}
