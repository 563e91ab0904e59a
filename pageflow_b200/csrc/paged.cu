// On-arrival decode of compressed column pages fused with a range filter and
// the first radix-partition pass (the paged path of the reference:
// IO/transfer/tick_layout.py:141-190 H2D pack + nvCOMP decompress, then
// pre_comp_stage mask compaction, then partition_sort; here one pipeline).
//
// The table arrives as PFC1 pages (codec.h) in pinned host memory, row group
// by row group (every column's page of rows [g*rpp, (g+1)*rpp), in column
// order).  Batches of row groups are copied to the device on a copy stream,
// up to NSTAGE batches ahead, while the compute stream runs per batch:
//   k_paged_hist     decode the filter and key columns of a quarter row group
//                    per CTA, count the passing rows per bucket
//   k_fscan-like     per bucket, each CTA's offset; bucket totals
//   k_paged_place    the batch's place in the output (a device cursor) and
//                    its bucket starts
//   k_paged_scatter  decode every column again, write each passing row's
//                    non-filter columns at its bucket's next slot
// No host wait happens inside the pipeline: the output cursor lives on the
// device, and a batch that would not fit the output capacity is skipped and
// flagged (stats[1]).  Decoding never goes through an intermediate buffer:
// compressed bytes are read once per pass, decoded in registers.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "codec.h"
#include "scan.cuh"

namespace pf {
namespace {

constexpr int QT = 512;              // threads of a decode CTA
constexpr int QV = 8;                // rows a thread per sub-tile (blocked)
constexpr int QSUB = QT * QV;        // 4096 rows: four PFC blocks
constexpr int QPARTS = 4;            // CTAs per row group
constexpr int MAXPC = 8;             // columns
constexpr int NSTAGE = 3;

struct PagedArgs {
  const uint8_t* stage;        // this batch's bytes
  const long long* dir;        // [n_groups][ncols] host byte offsets of the pages
  long long batch_start;       // host byte offset of the batch
  long long g0, g1;            // the batch's row groups
  int ncols, rpp;
  long long n_rows;
  int filter_col, key_col;
  long long lo, hi;            // filter: lo <= value < hi
  int B, logB;
  int* hist;                   // [ctas][B]
  const long long* boff;       // [B] this batch's bucket starts in the output
  void* outs[MAXPC];
  int esize[MAXPC];
  unsigned long long* stats;   // [0] rows out, [1] batches skipped, [2] bad pages
  const int* skip;             // this batch was skipped (no room)
};

__device__ __forceinline__ const uint8_t* page_of(const PagedArgs& a, long long g, int c) {
  return a.stage + (a.dir[g * a.ncols + c] - a.batch_start);
}

// The sub-tile's rows [r0, r0 + QSUB) of a FOR / DELTA stream, thread t's
// values at r0 + QV*t + k (zero past n).  DELTA scans each 1024-row mini-block
// (128 threads, four warps) from the block's first value.
__device__ void decode_stream_tile(const PfcStream* s, uint32_t r0, uint32_t n, int64_t (&out)[QV],
                                   long long* wsum) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint32_t j0 = r0 + QV * t;
  if (s->scheme == PFC_FOR) {
#pragma unroll
    for (int k = 0; k < QV; ++k) out[k] = j0 + k < n ? pfc_for_value(s, j0 + k) : 0;
    return;
  }
  long long run = 0;
#pragma unroll
  for (int k = 0; k < QV; ++k) {
    run += j0 + k < n ? pfc_delta_term(s, j0 + k) : 0;
    out[k] = run;
  }
  long long incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  long long pre = incl - run;
  const int seg0 = (w / 4) * 4;  // the first warp of this 1024-row block
  for (int q = seg0; q < w; ++q) pre += wsum[q];
#pragma unroll
  for (int k = 0; k < QV; ++k) out[k] += pre;
  __syncthreads();
}

// RLE pages: the page's runs (values, exclusive ends) staged in shared memory.
struct RunStage {
  long long vals[PFC_RLE_MAX_RUNS];
  long long ends[PFC_RLE_MAX_RUNS];
};

__device__ void stage_runs(const uint8_t* page, RunStage& rs, long long* wsum) {
  const PfcPage* h = (const PfcPage*)page;
  const PfcStream* sv = pfc_stream(page, h->s0);
  const PfcStream* se = pfc_stream(page, h->s1);
  int64_t v[QV];
  // runs <= PFC_RLE_MAX_RUNS == QSUB: one tile per stream
  decode_stream_tile(sv, 0, h->nruns, v, wsum);
#pragma unroll
  for (int k = 0; k < QV; ++k) {
    const uint32_t j = QV * threadIdx.x + k;
    if (j < h->nruns) rs.vals[j] = v[k];
  }
  decode_stream_tile(se, 0, h->nruns, v, wsum);
#pragma unroll
  for (int k = 0; k < QV; ++k) {
    const uint32_t j = QV * threadIdx.x + k;
    if (j < h->nruns) rs.ends[j] = v[k];
  }
  __syncthreads();
}

// The values of rows [r0, r0 + QSUB) of a page (blocked: thread t has QV*t..).
// An RLE page's runs are staged in rs first unless rs already holds them
// (*staged, the same for every thread).
__device__ void decode_page_tile(const uint8_t* page, uint32_t r0, int64_t (&out)[QV],
                                 RunStage* rs, const uint8_t** staged, long long* wsum) {
  const PfcPage* h = (const PfcPage*)page;
  if (h->scheme == PFC_RLE && *staged != page) {
    __syncthreads();  // every thread is done with the runs staged before
    stage_runs(page, *rs, wsum);
    *staged = page;
  }
  const uint32_t n = h->n, j0 = r0 + QV * threadIdx.x;
  switch (h->scheme) {
    case PFC_RAW:
#pragma unroll
      for (int k = 0; k < QV; ++k) {
        const uint32_t j = j0 + k;
        out[k] = j < n ? (h->esize == 8 ? ((const int64_t*)(page + h->s0))[j]
                                        : (int64_t)((const int32_t*)(page + h->s0))[j])
                       : 0;
      }
      break;
    case PFC_RLE: {
      // first run ending past j0, then walk
      int lo = 0, hi = (int)h->nruns - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (rs->ends[mid] > (long long)j0) hi = mid;
        else lo = mid + 1;
      }
      int run = lo;
#pragma unroll
      for (int k = 0; k < QV; ++k) {
        const uint32_t j = j0 + k;
        while (run + 1 < (int)h->nruns && rs->ends[run] <= (long long)j) ++run;
        out[k] = j < n ? rs->vals[run] : 0;
      }
      break;
    }
    default:
      decode_stream_tile(pfc_stream(page, h->s0), r0, n, out, wsum);
      break;
  }
}

struct QSmem {
  RunStage rs;          // the filter column's runs when it is RLE
  int cnt[4096];        // bucket counts / running slots
  long long wsum[QT / 32];
  int flag;
};

__device__ __forceinline__ bool page_ok(const uint8_t* page, int esize) {
  const PfcPage* h = (const PfcPage*)page;
  return h->magic == PFC_MAGIC && h->esize == esize && h->scheme <= PFC_RLE &&
         (h->scheme != PFC_RLE || h->nruns <= PFC_RLE_MAX_RUNS);
}

template <bool SCATTER>
__global__ void __launch_bounds__(QT) k_paged(PagedArgs a) {
  extern __shared__ __align__(16) unsigned char qsm[];
  QSmem& S = *reinterpret_cast<QSmem*>(qsm);
  if (SCATTER && *a.skip) return;
  const long long g = a.g0 + blockIdx.x / QPARTS;
  const int part = blockIdx.x % QPARTS;
  const long long grow0 = g * a.rpp;
  const int rows_g = (int)min((long long)a.rpp, a.n_rows - grow0);
  const int per = (a.rpp / QPARTS + QSUB - 1) / QSUB * QSUB;
  const int r_lo = part * per, r_hi = min(rows_g, r_lo + per);
  const int* hrow = a.hist + (long long)blockIdx.x * a.B;
  for (int b = threadIdx.x; b < a.B; b += QT) S.cnt[b] = 0;
  if (threadIdx.x == 0) {
    int bad = 0;
    for (int c = 0; c < a.ncols; ++c) bad |= !page_ok(page_of(a, g, c), a.esize[c]);
    S.flag = bad;
  }
  __syncthreads();
  if (S.flag) {
    if (threadIdx.x == 0 && !SCATTER) atomicAdd(&a.stats[2], 1ULL);
    if (!SCATTER)
      for (int b = threadIdx.x; b < a.B; b += QT) a.hist[(long long)blockIdx.x * a.B + b] = 0;
    return;
  }
  const uint8_t* fpage = page_of(a, g, a.filter_col);
  const uint8_t* staged = nullptr;
  unsigned long long out_rows = 0;
  for (int r0 = r_lo; r0 < r_hi; r0 += QSUB) {
    int64_t fv[QV], kv[QV];
    decode_page_tile(fpage, r0, fv, &S.rs, &staged, S.wsum);
    bool pass[QV], any = false;
#pragma unroll
    for (int k = 0; k < QV; ++k) {
      const int j = r0 + QV * threadIdx.x + k;
      pass[k] = j < r_hi && fv[k] >= a.lo && fv[k] < a.hi;
      any |= pass[k];
    }
    // a sub-tile that keeps no row decodes nothing more (the filter column is
    // often sorted: whole pages fall outside the range)
    if (!__syncthreads_or(any)) continue;
    decode_page_tile(page_of(a, g, a.key_col), r0, kv, &S.rs, &staged, S.wsum);
    int bk[QV];
#pragma unroll
    for (int k = 0; k < QV; ++k)
      bk[k] = pass[k] ? bucket_of_hash(mix64((uint64_t)kv[k]), a.logB) : -1;
    if (!SCATTER) {
#pragma unroll
      for (int k = 0; k < QV; ++k)
        if (bk[k] >= 0) atomicAdd(&S.cnt[bk[k]], 1);
      continue;
    }
    long long pos[QV];
#pragma unroll
    for (int k = 0; k < QV; ++k)
      pos[k] = bk[k] >= 0 ? a.boff[bk[k]] + hrow[bk[k]] + atomicAdd(&S.cnt[bk[k]], 1) : -1;
    for (int c = 0; c < a.ncols; ++c) {
      if (c == a.filter_col || !a.outs[c]) continue;
      int64_t v[QV];
      if (c == a.key_col) {
#pragma unroll
        for (int k = 0; k < QV; ++k) v[k] = kv[k];
      } else {
        decode_page_tile(page_of(a, g, c), r0, v, &S.rs, &staged, S.wsum);
      }
#pragma unroll
      for (int k = 0; k < QV; ++k) {
        if (pos[k] < 0) continue;
        if (a.esize[c] == 8) ((long long*)a.outs[c])[pos[k]] = v[k];
        else ((int*)a.outs[c])[pos[k]] = (int)v[k];
      }
    }
#pragma unroll
    for (int k = 0; k < QV; ++k) out_rows += pos[k] >= 0;
  }
  if (!SCATTER) {
    __syncthreads();
    for (int b = threadIdx.x; b < a.B; b += QT) a.hist[(long long)blockIdx.x * a.B + b] = S.cnt[b];
  } else {
    for (int o = 16; o; o >>= 1) out_rows += __shfl_xor_sync(FULL, out_rows, o);
    if ((threadIdx.x & 31) == 0 && out_rows) atomicAdd(&a.stats[0], out_rows);
  }
}

// Per bucket, each CTA's offset inside the batch's bucket run; counts[b].
__global__ void __launch_bounds__(512) k_paged_scan(int* __restrict__ hist, int nctas, int B,
                                                   long long* __restrict__ counts) {
  constexpr int W = 16;
  __shared__ long long part[W][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * 32 + lane;
  const bool live = b < B;
  const int per = (nctas + W - 1) / W;
  const int c0 = w * per, c1 = min(nctas, c0 + per);
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

// The batch's place: its bucket starts in the output after the rows already
// placed (the device cursor), or a skip flag when it would not fit.
// bucket_offsets row of the batch: [B] starts, [B] the batch's total.
__global__ void __launch_bounds__(1024) k_paged_place(const long long* __restrict__ counts, int B,
                                                      unsigned long long* cursor,
                                                      long long capacity, long long* boff,
                                                      long long* row_out, int* skip,
                                                      unsigned long long* stats) {
  __shared__ long long wsum[32];
  __shared__ long long base;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int per = (B + 1023) / 1024;
  long long s = 0;
  for (int q = 0; q < per; ++q) {
    const int b = tid * per + q;
    if (b < B) s += counts[b];
  }
  long long incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (tid == 0) {
    long long tot = 0;
    for (int q = 0; q < 32; ++q) {
      const long long t = wsum[q];
      wsum[q] = tot;
      tot += t;
    }
    const unsigned long long b0 = atomicAdd(cursor, (unsigned long long)tot);
    if ((long long)b0 + tot > capacity) {
      *skip = 1;
      atomicAdd(cursor, (unsigned long long)(-tot));
      atomicAdd(&stats[1], 1ULL);
      base = -1;
    } else {
      *skip = 0;
      base = (long long)b0;
    }
    row_out[B] = tot;
  }
  __syncthreads();
  long long ex = wsum[w] + incl - s;
  for (int q = 0; q < per; ++q) {
    const int b = tid * per + q;
    if (b < B) {
      boff[b] = base < 0 ? 0 : base + ex;
      row_out[b] = base < 0 ? -1 : base + ex;
      ex += counts[b];
    }
  }
}

struct PagedLayout {
  uint8_t* stage[NSTAGE];
  long long* dir;
  int* hist;
  long long* counts;
  long long* boff;
  int* skip;
  unsigned long long* cursor;
};

PagedLayout paged_layout(Arena& a, long long max_batch_bytes, long long n_dir, int ctas, int B) {
  PagedLayout l{};
  for (int s = 0; s < NSTAGE; ++s) l.stage[s] = a.take<uint8_t>(std::max<long long>(max_batch_bytes, 16));
  l.dir = a.take<long long>(std::max<long long>(n_dir, 1));
  l.hist = a.take<int>((size_t)ctas * B);
  l.counts = a.take<long long>(B);
  l.boff = a.take<long long>(B);
  l.skip = a.take<int>(NSTAGE);
  l.cursor = a.take<unsigned long long>(1);
  return l;
}

long long batch_bytes(const long long* dir, long long n_groups, int ncols, long long total,
                      long long g0, long long g1) {
  const long long s = dir[g0 * ncols];
  const long long e = g1 < n_groups ? dir[g1 * ncols] : total;
  return e - s;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_paged_scan_workspace(const int64_t* directory, int64_t n_groups, int ncols,
                                          int64_t total_bytes, int groups_per_batch, int B) {
  long long mx = 0;
  for (long long g0 = 0; g0 < n_groups; g0 += groups_per_batch)
    mx = std::max(mx, batch_bytes((const long long*)directory, n_groups, ncols, total_bytes, g0,
                                  std::min<long long>(n_groups, g0 + groups_per_batch)));
  Arena a(nullptr, 0);
  paged_layout(a, mx, n_groups * ncols, groups_per_batch * QPARTS, std::max(B, 1));
  return a.used + 256;
}

extern "C" int pf_paged_scan(const uint8_t* host_pages, const int64_t* directory, int64_t n_groups,
                             int ncols, const int* esizes, int64_t total_bytes, int64_t n_rows,
                             int rows_per_page, int filter_col, int64_t lo, int64_t hi,
                             int key_col, int B, int groups_per_batch, void* const* outs,
                             int64_t capacity_rows, int64_t* bucket_offsets, int64_t* stats,
                             void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ncols < 1 || ncols > MAXPC || filter_col < 0 || filter_col >= ncols || key_col < 0 ||
      key_col >= ncols || key_col == filter_col)
    return fail(PF_EINVAL, "paged_scan: bad columns");
  if (B < 1 || B > 4096 || (B & (B - 1))) return fail(PF_EINVAL, "paged_scan: B must be a power of two <= 4096");
  if (rows_per_page < QSUB || rows_per_page % (QSUB * QPARTS))
    return fail(PF_EINVAL, "paged_scan: rows_per_page must be a multiple of %d", QSUB * QPARTS);
  if (groups_per_batch < 1 || n_groups < 1 || n_rows > n_groups * (int64_t)rows_per_page)
    return fail(PF_EINVAL, "paged_scan: bad sizes");
  if (esizes[key_col] != 8) return fail(PF_EINVAL, "paged_scan: the key column must be int64");
  long long mx = 0;
  const long long* dir = (const long long*)directory;
  for (long long g0 = 0; g0 < n_groups; g0 += groups_per_batch)
    mx = std::max(mx, batch_bytes(dir, n_groups, ncols, total_bytes, g0,
                                  std::min<long long>(n_groups, g0 + groups_per_batch)));
  Arena ar(workspace, workspace_bytes);
  PagedLayout l = paged_layout(ar, mx, n_groups * ncols, groups_per_batch * QPARTS, B);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "paged_scan: workspace of %zu bytes, %zu needed", workspace_bytes, ar.used);

  // the copy stream and the events of this thread and device
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  struct Res {
    cudaStream_t copy;
    cudaEvent_t copied[NSTAGE], freed[NSTAGE];
  };
  thread_local std::map<int, Res> resources;
  auto it = resources.find(dev);
  if (it == resources.end()) {
    Res r{};
    PF_CUDA(cudaStreamCreateWithFlags(&r.copy, cudaStreamNonBlocking));
    for (int s = 0; s < NSTAGE; ++s) {
      PF_CUDA(cudaEventCreateWithFlags(&r.copied[s], cudaEventDisableTiming));
      PF_CUDA(cudaEventCreateWithFlags(&r.freed[s], cudaEventDisableTiming));
    }
    it = resources.emplace(dev, r).first;
  }
  Res& R = it->second;

  PF_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(int64_t), st));
  PF_CUDA(cudaMemsetAsync(l.cursor, 0, sizeof(unsigned long long), st));
  PF_CUDA(cudaMemcpyAsync(l.dir, directory, sizeof(long long) * n_groups * ncols,
                          cudaMemcpyHostToDevice, st));
  // the copy stream starts after the stream's work so far
  cudaEvent_t start_ev;
  if (int rc = record_event(st, &start_ev)) return rc;
  PF_CUDA(cudaStreamWaitEvent(R.copy, start_ev, 0));

  PagedArgs a{};
  a.dir = l.dir;
  a.ncols = ncols;
  a.rpp = rows_per_page;
  a.n_rows = n_rows;
  a.filter_col = filter_col;
  a.key_col = key_col;
  a.lo = lo;
  a.hi = hi;
  a.B = B;
  a.logB = log2_exact((uint64_t)B);
  a.hist = l.hist;
  a.boff = l.boff;
  for (int c = 0; c < ncols; ++c) {
    a.outs[c] = outs[c];
    a.esize[c] = esizes[c];
  }
  a.stats = (unsigned long long*)stats;
  const size_t smem = sizeof(QSmem);
  if (int rc = opt_in_smem((const void*)k_paged<false>, smem)) return rc;
  if (int rc = opt_in_smem((const void*)k_paged<true>, smem)) return rc;
  const long long nb = (n_groups + groups_per_batch - 1) / groups_per_batch;
  for (long long k = 0; k < nb; ++k) {
    const int s = (int)(k % NSTAGE);
    const long long g0 = k * groups_per_batch, g1 = std::min<long long>(n_groups, g0 + groups_per_batch);
    const long long bs = dir[g0 * ncols];
    const long long bytes = batch_bytes(dir, n_groups, ncols, total_bytes, g0, g1);
    if (k >= NSTAGE) PF_CUDA(cudaStreamWaitEvent(R.copy, R.freed[s], 0));
    PF_CUDA(cudaMemcpyAsync(l.stage[s], host_pages + bs, bytes, cudaMemcpyHostToDevice, R.copy));
    PF_CUDA(cudaEventRecord(R.copied[s], R.copy));
    PF_CUDA(cudaStreamWaitEvent(st, R.copied[s], 0));
    a.stage = l.stage[s];
    a.batch_start = bs;
    a.g0 = g0;
    a.g1 = g1;
    a.skip = l.skip + s;
    const int ctas = (int)(g1 - g0) * QPARTS;
    {
      PF_KERNEL("k_paged_hist", st);
      k_paged<false><<<ctas, QT, smem, st>>>(a);
    }
    {
      PF_KERNEL("k_paged_scan", st);
      k_paged_scan<<<(B + 31) / 32, 512, 0, st>>>(l.hist, ctas, B, l.counts);
    }
    {
      PF_KERNEL("k_paged_place", st);
      k_paged_place<<<1, 1024, 0, st>>>(l.counts, B, l.cursor, capacity_rows, l.boff,
                                        (long long*)bucket_offsets + k * (B + 1), l.skip + s,
                                        (unsigned long long*)stats);
    }
    {
      PF_KERNEL("k_paged_scatter", st);
      k_paged<true><<<ctas, QT, smem, st>>>(a);
    }
    PF_CUDA(cudaEventRecord(R.freed[s], st));
  }
  PF_LAUNCH("k_paged");
  return ok();
}
