// Serving: join -> date filter -> group-by requests against resident
// dimension tables, folded into persistent launches.
//
// A dimension table's hash table is built once (pf_dim_build) and stays in
// HBM across requests: 16-byte slots {key, OCCUPIED | group}, a power of two
// of at least twice its keys, linear probing from the multiply-shift of the
// key's mix64.  A slot is claimed by a CAS of its second word from zero, then
// its key is stored; probes run in later launches only.
//
// pf_serve_run runs one launch over a list of requests, each a range of its
// probe rows [row_begin, row_end) and, for a request's last launch, its
// finish.  Work items, request by request in the order given:
//   probe items   PROBE_ROWS rows each: keep date in [lo, hi), look the FK up,
//                 add (value, 1) into the request's (sum, count) slab with
//                 warp-combined REDs
//   count items   (finish) GROUP_CHUNK groups each: occupied groups, after
//                 the request's probe items of this launch are done
//   emit items    (finish) the chunk's occupied groups in ascending order at
//                 the chunk's offset, after the count items are done; the
//                 last one writes the group count and sets the request's
//                 pinned done word to 1 + groups (~0 if a wait gave up)
// A block takes the next item from one counter; a finish item waits
// (bounded) for items of its own request that were taken before it by
// blocks that are running, so every wait ends.  The host sees a request
// complete through its done word while the launch goes on with others.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>

#include "agg.cuh"

namespace pf {
namespace {

constexpr int ST = 256;
#ifndef PF_SERVE_SV
#define PF_SERVE_SV 2
#endif
// 1: the probe loop loads the next round's dates while this round runs;
// 2: its keys too, filtered or not (the kernel is bound by its dependent
// loads, not by bytes: with 2 rows a thread, 91.1 against 85.4 G rows/s for
// dates only at 4 rows a thread, saturated)
#ifndef PF_SERVE_PIPE
#define PF_SERVE_PIPE 2
#endif
constexpr int SV = PF_SERVE_SV;  // probe rows a thread keeps in flight
// 1: probe items add through the block's group cache (agg.cuh), flushed at
// the item's end; 0: hot_add into the slab directly.
#ifndef PF_SERVE_CACHE
#define PF_SERVE_CACHE 1
#endif
constexpr size_t SERVE_CACHE_SMEM = PF_SERVE_CACHE ? sizeof(GroupCache) : 0;
constexpr long long PROBE_ROWS = 16384;
constexpr long long GROUP_CHUNK = 16384;
constexpr long long MAX_CHUNKS = 256;  // groups <= 4M a request
constexpr unsigned WAIT_LIMIT = 1u << 22;
constexpr int MAX_REQUESTS = 8192;  // a launch's requests (their first items sit in smem)
constexpr unsigned long long OCCUPIED = 1ULL << 63;
constexpr unsigned long long NO_GROUP = 0xffffffffULL;

struct DimSlot {
  unsigned long long key;
  unsigned long long val;  // OCCUPIED | group (NO_GROUP: outside [0, n_groups))
};

__device__ __forceinline__ unsigned long long dim_first_slot(uint64_t h, int logcap) {
  return h >> (64 - logcap);
}

__global__ void __launch_bounds__(256) k_dim_build(const long long* __restrict__ keys,
                                                   const int* __restrict__ groups, long long n,
                                                   long long n_groups, DimSlot* table,
                                                   int logcap,
                                                   unsigned long long* __restrict__ stats) {
  const unsigned long long mask = (1ULL << logcap) - 1;
  unsigned long long bad = 0, overflow = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)keys[i];
    const int g = groups[i];
    unsigned long long v = OCCUPIED | (unsigned long long)(unsigned)g;
    if (g < 0 || (long long)g >= n_groups) {
      v = OCCUPIED | NO_GROUP;
      ++bad;
    }
    unsigned long long s = dim_first_slot(mix64(key), logcap);
    bool done = false;
    for (unsigned long long probes = 0; probes <= mask; ++probes) {
      if (atomicCAS(&table[s].val, 0ULL, v) == 0ULL) {
        table[s].key = key;
        done = true;
        break;
      }
      s = (s + 1) & mask;
    }
    overflow += !done;
  }
  if (bad) atomicAdd(&stats[0], bad);
  if (overflow) atomicAdd(&stats[1], overflow);
}

struct SReq {
  const long long* fk;
  const int* date;
  const long long* value;
  long long r0, r1;
  const DimSlot* table;
  long long ng;
  unsigned long long* slab;
  long long* okeys;
  long long* osums;
  long long* ocounts;
  long long* on;
  unsigned long long* done;  // device alias of the pinned done word, or null
  long long item0, npi, nch;  // first item; probe items; finish chunks (0: no finish)
  int lo, hi;
  int logcap;
  int pad;
};

struct SCounters {
  unsigned probe_left, count_left, emit_left, pad;
};

struct SHead {
  unsigned long long counter;
  long long n_items;
  int n_req;
  int pad;
  unsigned long long error;
};

// The request of item `it`: the last request whose first item is <= it
// (first[] holds every request's first item, in shared memory).
__device__ __forceinline__ int request_of(const int* first, int n, long long it) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= it) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void set_done(unsigned long long* done, unsigned long long v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(done), "l"(v) : "memory");
}

// Thread 0 waits (bounded) until *left is zero; false when it gave up, after
// raising the error word and marking the request's done word failed (~0).
__device__ bool wait_zero(const unsigned* left, SHead* h, unsigned long long* done) {
  unsigned polls = 0;
  while (ld_acquire_u32(left) != 0 && polls < WAIT_LIMIT) {
    __nanosleep(200);
    ++polls;
  }
  if (polls >= WAIT_LIMIT) {
    atomicOr(&h->error, 1ULL);
    if (done) set_done(done, ~0ULL);
    return false;
  }
  __threadfence();
  return true;
}

__device__ __forceinline__ long long block_sum(long long v, long long* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  long long t = 0;
  for (int q = 0; q < ST / 32; ++q) t += red[q];
  return t;
}

__global__ void __launch_bounds__(ST) k_serve(SHead* h, const SReq* __restrict__ reqs,
                                              SCounters* cnt, long long* chunk_counts,
                                              unsigned long long* stats) {
  extern __shared__ __align__(16) unsigned char serve_smem[];
  GroupCache& gc = *reinterpret_cast<GroupCache*>(serve_smem);
  int* first_item = reinterpret_cast<int*>(serve_smem + SERVE_CACHE_SMEM);
  if (PF_SERVE_CACHE) cache_init(gc);
  __shared__ long long item_s;
  __shared__ int ok_s;
  __shared__ long long red[ST / 32];
  __shared__ int wpre[ST / 32];
  const long long ni = h->n_items;
  const int n = h->n_req;
  for (int i = threadIdx.x; i < n; i += ST) first_item[i] = (int)reqs[i].item0;
  unsigned long long matched = 0, kept = 0;
  long long hot = -1;  // the warp's hot group (hot_add)
  // With PF_PREFETCH_ITEMS, thread 0 takes the block's next item while the
  // block works on the current one (measured no faster, so off by default).
  // Items are taken in increasing order and an item waits only for items
  // before it, so the smallest unfinished item is always some block's
  // current item with nothing left to wait for: the launch progresses.
  if (threadIdx.x == 0) item_s = (long long)atomicAdd(&h->counter, 1ULL);
  while (true) {
    __syncthreads();
    const long long it = item_s;
    if (it >= ni) break;
    unsigned long long next = 0;
    if (PF_PREFETCH_ITEMS && threadIdx.x == 0) next = atomicAdd(&h->counter, 1ULL);
    const int q = request_of(first_item, n, it);
    const SReq& R = reqs[q];
    const long long local = it - R.item0;
    if (local < R.npi) {
      // ---- probe rows, SV a thread at a time: every stage (dates, keys, first
      // slots, values) is issued for all SV rows before any is used, so a
      // thread keeps SV independent loads in flight
      const long long lo = R.r0 + local * PROBE_ROWS, hi = min(R.r1, lo + PROBE_ROWS);
      const unsigned long long mask = (1ULL << R.logcap) - 1;
#if PF_SERVE_PIPE
      // the next round's dates (and, with PF_SERVE_PIPE 2, its keys, whether
      // the rows pass the filter or not) load while this round runs
      int dt[SV];
      unsigned long long kf[PF_SERVE_PIPE >= 2 ? SV : 1];
#pragma unroll
      for (int k = 0; k < SV; ++k) {
        const long long i = lo + k * ST + threadIdx.x;
        dt[k] = i < hi ? R.date[i] : INT_MIN;
        if (PF_SERVE_PIPE >= 2) kf[k < SV ? k : 0] = i < hi ? (unsigned long long)R.fk[i] : 0ULL;
      }
#endif
      for (long long i0 = lo; i0 < hi; i0 += ST * SV) {
        bool keep[SV];
        unsigned long long key[SV], slot[SV];
        ulonglong2 sl[SV];
        long long g[SV], value[SV];
#if PF_SERVE_PIPE
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          keep[k] = dt[k] >= R.lo && dt[k] < R.hi;
          if (PF_SERVE_PIPE >= 2) key[k] = keep[k] ? kf[k < SV ? k : 0] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          const long long i = i0 + (long long)ST * SV + k * ST + threadIdx.x;
          dt[k] = i < hi ? R.date[i] : INT_MIN;
          if (PF_SERVE_PIPE >= 2) kf[k < SV ? k : 0] = i < hi ? (unsigned long long)R.fk[i] : 0ULL;
        }
#else
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          const long long i = i0 + k * ST + threadIdx.x;
          const int d = i < hi ? R.date[i] : INT_MIN;
          keep[k] = d >= R.lo && d < R.hi;
        }
#endif
#pragma unroll
        for (int k = 0; k < (PF_SERVE_PIPE >= 2 ? 0 : SV); ++k) {
          const long long i = i0 + k * ST + threadIdx.x;
          key[k] = keep[k] ? (unsigned long long)R.fk[i] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          slot[k] = dim_first_slot(mix64(key[k]), R.logcap);
          sl[k] = keep[k] ? *reinterpret_cast<const ulonglong2*>(R.table + slot[k])
                          : make_ulonglong2(0ULL, 0ULL);
        }
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          g[k] = -1;
          if (!keep[k]) continue;
          ++kept;
          unsigned long long sk = slot[k];
          ulonglong2 x = sl[k];
          for (unsigned long long probes = 0; probes <= mask; ++probes) {
            if (x.y == 0) break;
            if (x.x == key[k]) {
              ++matched;
              const unsigned long long go = x.y & ~OCCUPIED;
              if (go != NO_GROUP) g[k] = (long long)go;
              break;
            }
            sk = (sk + 1) & mask;
            x = *reinterpret_cast<const ulonglong2*>(R.table + sk);
          }
        }
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          const long long i = i0 + k * ST + threadIdx.x;
          value[k] = g[k] >= 0 ? R.value[i] : 0;
        }
#pragma unroll
        for (int k = 0; k < SV; ++k) {
          if (PF_SERVE_CACHE) {
            if (g[k] >= 0) cache_add(gc, R.slab, g[k], (unsigned long long)value[k], 1ULL);
          } else {
            hot_add(R.slab, g[k], value[k], hot);
          }
        }
      }
      if (PF_SERVE_CACHE) cache_flush(gc, R.slab);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicSub(&cnt[q].probe_left, 1u);
      }
    } else if (local < R.npi + R.nch) {
      // ---- count a chunk's occupied groups
      const long long c = local - R.npi;
      if (threadIdx.x == 0) ok_s = wait_zero(&cnt[q].probe_left, h, R.done);
      __syncthreads();
      if (!ok_s) {
        if (threadIdx.x == 0) item_s = (long long)(PF_PREFETCH_ITEMS ? next : atomicAdd(&h->counter, 1ULL));
        continue;
      }
      const long long g0 = c * GROUP_CHUNK, g1 = min(R.ng, g0 + GROUP_CHUNK);
      long long occ = 0;
      for (long long g = g0 + threadIdx.x; g < g1; g += ST) occ += __ldcg(&R.slab[2 * g + 1]) != 0;
      occ = block_sum(occ, red);
      if (threadIdx.x == 0) {
        chunk_counts[(long long)q * MAX_CHUNKS + c] = occ;
        __threadfence();
        atomicSub(&cnt[q].count_left, 1u);
      }
    } else {
      // ---- emit a chunk's occupied groups, ascending
      const long long c = local - R.npi - R.nch;
      if (threadIdx.x == 0) ok_s = wait_zero(&cnt[q].count_left, h, R.done);
      __syncthreads();
      if (!ok_s) {
        if (threadIdx.x == 0) item_s = (long long)(PF_PREFETCH_ITEMS ? next : atomicAdd(&h->counter, 1ULL));
        continue;
      }
      const long long* cc = chunk_counts + (long long)q * MAX_CHUNKS;
      long long base = 0, total = 0;
      for (long long k = 0; k < R.nch; ++k) {
        const long long v = __ldcg(&cc[k]);
        if (k < c) base += v;
        total += v;
      }
      const long long g0 = c * GROUP_CHUNK, g1 = min(R.ng, g0 + GROUP_CHUNK);
      const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      for (long long t0 = g0; t0 < g1; t0 += ST) {
        const long long g = t0 + threadIdx.x;
        unsigned long long s = 0, k = 0;
        if (g < g1) {
          s = __ldcg(&R.slab[2 * g]);
          k = __ldcg(&R.slab[2 * g + 1]);
        }
        const bool occ = k != 0;
        const unsigned bal = __ballot_sync(FULL, occ);
        __syncthreads();
        if (lane == 0) wpre[w] = __popc(bal);
        __syncthreads();
        int before = 0, tile = 0;
        for (int qw = 0; qw < ST / 32; ++qw) {
          if (qw < w) before += wpre[qw];
          tile += wpre[qw];
        }
        if (occ) {
          const long long o = base + before + __popc(bal & ((1u << lane) - 1));
          R.okeys[o] = g;
          R.osums[o] = (long long)s;
          R.ocounts[o] = (long long)k;
        }
        base += tile;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        if (atomicSub(&cnt[q].emit_left, 1u) == 1u) {
          *R.on = total;
          __threadfence_system();
          if (R.done) set_done(R.done, (unsigned long long)(total + 1));
        }
      }
    }
    __syncthreads();  // every thread has read item_s
    if (threadIdx.x == 0) item_s = (long long)(PF_PREFETCH_ITEMS ? next : atomicAdd(&h->counter, 1ULL));
  }
  for (int o = 16; o; o >>= 1) {
    matched += __shfl_xor_sync(FULL, matched, o);
    kept += __shfl_xor_sync(FULL, kept, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (matched) atomicAdd(&stats[0], matched);
    if (kept) atomicAdd(&stats[2], kept);
  }
}

__global__ void k_serve_error(const SHead* h, unsigned long long* stats) {
  if (threadIdx.x == 0 && h->error) stats[1] |= h->error;
}

struct ServeLayout {
  SHead* head;
  SReq* reqs;
  SCounters* cnt;
  long long* chunks;
};

ServeLayout serve_layout(Arena& a, int n) {
  ServeLayout l{};
  l.head = a.take<SHead>(1);
  l.reqs = a.take<SReq>(std::max(n, 1));
  l.cnt = a.take<SCounters>(std::max(n, 1));
  l.chunks = a.take<long long>((size_t)std::max(n, 1) * MAX_CHUNKS);
  return l;
}

// The host image of a launch's header, requests and counters is written into
// pinned staging (one per device and host thread) and copied in one piece;
// the staging is reused once the previous copy out of it has completed.
struct Staging {
  char* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  bool pending = false;
};

int staging_for(size_t bytes, Staging** out) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  thread_local std::map<int, Staging> stages;
  Staging& s = stages[dev];
  if (!s.ev) PF_CUDA(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  if (s.pending) {
    if (int rc = wait_event(s.ev)) return rc;
    s.pending = false;
  }
  if (s.cap < bytes) {
    if (s.buf) PF_CUDA(cudaFreeHost(s.buf));
    s.buf = nullptr;
    s.cap = 0;
    const size_t want = std::max<size_t>(bytes * 2, 1 << 16);
    PF_CUDA(cudaHostAlloc((void**)&s.buf, want, cudaHostAllocDefault));
    s.cap = want;
  }
  *out = &s;
  return PF_OK;
}

int serve_grid(int* grid, size_t smem) {
  int per_sm = 0;
  if (int rc = opt_in_smem((const void*)k_serve, smem)) return rc;
  PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_serve, ST, smem));
  *grid = std::max(1, per_sm) * sm_count();
  return PF_OK;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_dim_table_bytes(int64_t n_keys) {
  const uint64_t cap = pow2_at_least((uint64_t)std::max<int64_t>(2 * n_keys, 2));
  return (size_t)cap * sizeof(DimSlot);
}

extern "C" int pf_dim_build(const int64_t* keys, const int32_t* groups, int64_t n_keys,
                            int64_t n_groups, void* table, size_t table_bytes, int64_t* stats,
                            void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n_keys < 1 || n_groups < 1 || n_groups >= (int64_t)NO_GROUP)
    return fail(PF_EINVAL, "dim_build: bad sizes");
  if (!keys || !groups || !table || !stats) return fail(PF_EINVAL, "dim_build: null pointer");
  const size_t need = pf_dim_table_bytes(n_keys);
  if (table_bytes < need)
    return fail(PF_ENOSPACE, "dim_build: table of %zu bytes, %zu needed", table_bytes, need);
  const uint64_t cap = need / sizeof(DimSlot);
  PF_CUDA(cudaMemsetAsync(table, 0, need, st));
  PF_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(int64_t), st));
  const unsigned grid = (unsigned)std::max<long long>(
      1, std::min<long long>((n_keys + 255) / 256, (long long)sm_count() * 16));
  {
    PF_KERNEL("k_dim_build", st);
    k_dim_build<<<grid, 256, 0, st>>>((const long long*)keys, groups, n_keys, n_groups,
                                      (DimSlot*)table, log2_exact(cap),
                                      (unsigned long long*)stats);
  }
  PF_LAUNCH("k_dim_build");
  return ok();
}

extern "C" size_t pf_serve_workspace(int max_requests) {
  Arena a(nullptr, 0);
  serve_layout(a, max_requests);
  return a.used + 256;
}

extern "C" int pf_serve_run(const pf_serve_request* reqs, int n, void* workspace,
                            size_t workspace_bytes, int64_t* stats, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 1 || n > MAX_REQUESTS)
    return fail(PF_EINVAL, "serve_run: 1 to %d requests a launch, got %d", MAX_REQUESTS, n);
  if (!stats) return fail(PF_EINVAL, "serve_run: null stats");
  Arena a(workspace, workspace_bytes);
  ServeLayout l = serve_layout(a, n);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "serve_run: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  // one host image of header, requests and counters, copied in one piece
  const size_t off_r = (char*)l.reqs - (char*)l.head, off_c = (char*)l.cnt - (char*)l.head;
  const size_t bytes = off_c + sizeof(SCounters) * n;
  Staging* stg = nullptr;
  if (int rc = staging_for(bytes, &stg)) return rc;
  char* img = stg->buf;
  std::memset(img, 0, bytes);
  SHead* H = (SHead*)img;
  SReq* D = (SReq*)(img + off_r);
  SCounters* C = (SCounters*)(img + off_c);
  long long items = 0;
  for (int i = 0; i < n; ++i) {
    const pf_serve_request& x = reqs[i];
    if (!x.table || x.n_keys < 1 || x.n_groups < 1 || x.n_groups > GROUP_CHUNK * MAX_CHUNKS)
      return fail(PF_EINVAL, "serve_run: request %d: bad table or groups (at most %lld)", i,
                  (long long)(GROUP_CHUNK * MAX_CHUNKS));
    if (x.row_begin < 0 || x.row_end < x.row_begin)
      return fail(PF_EINVAL, "serve_run: request %d: bad row range", i);
    if (x.row_end > x.row_begin && (!x.fk || !x.date || !x.value))
      return fail(PF_EINVAL, "serve_run: request %d: null column", i);
    if (!x.slab || (x.finish && (!x.out_keys || !x.out_sums || !x.out_counts || !x.out_n)))
      return fail(PF_EINVAL, "serve_run: request %d: null output", i);
    SReq& R = D[i];
    R.fk = (const long long*)x.fk;
    R.date = x.date;
    R.value = (const long long*)x.value;
    R.r0 = x.row_begin;
    R.r1 = x.row_end;
    R.table = (const DimSlot*)x.table;
    R.logcap = log2_exact(pf_dim_table_bytes(x.n_keys) / sizeof(DimSlot));
    R.ng = x.n_groups;
    R.slab = (unsigned long long*)x.slab;
    R.okeys = (long long*)x.out_keys;
    R.osums = (long long*)x.out_sums;
    R.ocounts = (long long*)x.out_counts;
    R.on = (long long*)x.out_n;
    R.done = nullptr;
    if (x.finish && x.done) {
      if (int rc = host_alias((void*)x.done, (void**)&R.done)) return rc;
    }
    R.lo = x.date_lo;
    R.hi = x.date_hi;
    if (items > INT_MAX / 2) return fail(PF_EINVAL, "serve_run: too many work items");
    R.item0 = items;
    R.npi = (x.row_end - x.row_begin + PROBE_ROWS - 1) / PROBE_ROWS;
    R.nch = x.finish ? (x.n_groups + GROUP_CHUNK - 1) / GROUP_CHUNK : 0;
    items += R.npi + 2 * R.nch;
    C[i].probe_left = (unsigned)R.npi;
    C[i].count_left = (unsigned)R.nch;
    C[i].emit_left = (unsigned)R.nch;
  }
  H->counter = 0;
  H->n_items = items;
  H->n_req = n;
  H->error = 0;
  int grid = 0;
  if (int rc = serve_grid(&grid, SERVE_CACHE_SMEM + sizeof(int) * n)) return rc;
  PF_CUDA(cudaMemcpyAsync(l.head, img, bytes, cudaMemcpyHostToDevice, st));
  PF_CUDA(cudaEventRecord(stg->ev, st));
  stg->pending = true;
  {
    PF_KERNEL("k_serve", st);
    k_serve<<<grid, ST, SERVE_CACHE_SMEM + sizeof(int) * n, st>>>(l.head, l.reqs, l.cnt, l.chunks,
                                                (unsigned long long*)stats);
  }
  PF_LAUNCH("k_serve");
  {
    PF_KERNEL("k_serve_error", st);
    k_serve_error<<<1, 32, 0, st>>>(l.head, (unsigned long long*)stats);
  }
  PF_LAUNCH("k_serve_error");
  return ok();
}
