// The sorted-run primitives of the two-pass aggregation (PageFlow's
// operators/sorted_run_merge.py) on sm_100a:
//
//   pf_sort_pairs        stable ascending sort of int64 keys with an int64
//                        payload: least-significant-digit radix sort, 8-bit
//                        digits of (key - min), only as many passes as the key
//                        range needs (one host wait for the range)
//   pf_unique_reduce     reduce_tick_slice (sorted_run_merge.py:62-92): the
//                        unique keys ascending and, per value column, the sum /
//                        max / min of each key's rows (include_self=False)
//   pf_merge_sorted_runs merge_sorted_unique_runs_inplace (:94-174): the union
//                        of two ascending unique runs, matched keys combined,
//                        out of place (the caller copies it back)
//
// A radix pass: k_rs_hist counts each 4096-key tile's digits; an exclusive
// scan over [digit][tile] gives every (digit, tile) run's output start;
// k_rs_scatter ranks each tile's keys stably - a key's rank among its warp's
// equal digits from __match_any_sync, the warps' counts prefixed per digit in
// shared memory - and writes them through a staged copy of the tile.
#include <algorithm>
#include <climits>
#include <map>

#include "scan.cuh"

namespace pf {
namespace {

constexpr int RT = 256;
constexpr int RITEMS = 16;
constexpr int RTILE = RT * RITEMS;

__global__ void k_minmax_init(long long* mm) {
  mm[0] = LLONG_MAX;
  mm[1] = LLONG_MIN;
}

__global__ void __launch_bounds__(RT) k_minmax(const long long* __restrict__ k, long long n,
                                               long long* mm) {
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (long long i = (long long)blockIdx.x * RT + threadIdx.x; i < n;
       i += (long long)gridDim.x * RT) {
    const long long v = k[i];
    lo = min(lo, v);
    hi = max(hi, v);
  }
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(FULL, lo, o));
    hi = max(hi, __shfl_xor_sync(FULL, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
}

__device__ __forceinline__ int digit_of(long long key, long long kmin, int shift) {
  return (int)((((unsigned long long)key - (unsigned long long)kmin) >> shift) & 255u);
}

__global__ void __launch_bounds__(RT) k_rs_hist(const long long* __restrict__ keys, long long n,
                                                long long kmin, int shift, int ntiles,
                                                long long* __restrict__ hist) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * RTILE;
  long long kv[RITEMS];
#pragma unroll
  for (int k = 0; k < RITEMS; ++k) {
    const long long i = t0 + k * RT + threadIdx.x;
    kv[k] = i < n ? keys[i] : 0;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < RITEMS; ++k)
    if (t0 + k * RT + threadIdx.x < n) atomicAdd(&h[digit_of(kv[k], kmin, shift)], 1);
  __syncthreads();
  hist[(long long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// 512 threads take a tile, each warp a contiguous 256-key segment (8 keys a
// lane, item k of lane l at w*256 + k*32 + l).  A key's place among its
// warp's equal digits comes from __match_any_sync, item by item; the warps'
// digit counts give every digit's run in the tile (digit order) and each
// warp's place inside it.  The keys are staged at their places in shared
// memory and written out digit run by digit run, consecutive threads on
// consecutive rows; then the values the same way through the same buffer
// (their loads issued before the keys' write-out).
constexpr int ST = 512;
constexpr int SI = RTILE / ST;  // keys a thread
constexpr int SW = ST / 32;
constexpr int SSEG = SI * 32;   // keys a warp
static_assert(ST >= 256, "a thread a digit");

struct ScatterSmem {
  long long stage[RTILE];
  int wh[SW][256];  // the warp's digit counts, then its place in the digit's run
  int tstart[256];  // the digit's first place in the tile
  long long gbase[256];
  unsigned char sdig[RTILE];
  int wsum[SW];
};

__global__ void __launch_bounds__(ST, 2) k_rs_scatter(const long long* __restrict__ kin,
                                                   const long long* __restrict__ vin, long long n,
                                                   long long kmin, int shift, int ntiles,
                                                   const long long* __restrict__ offsets,
                                                   long long* __restrict__ kout,
                                                   long long* __restrict__ vout) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  ScatterSmem& S = *reinterpret_cast<ScatterSmem*>(rs_smem);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int x = tid; x < SW * 256; x += ST) (&S.wh[0][0])[x] = 0;
  const long long t0 = (long long)blockIdx.x * RTILE;
  const long long s0 = t0 + (long long)w * SSEG + lane;
  long long key[SI];
  int dig[SI];
#pragma unroll
  for (int k = 0; k < SI; ++k) key[k] = s0 + k * 32 < n ? kin[s0 + k * 32] : 0;
  const long long goff = tid < 256 ? offsets[(long long)tid * ntiles + blockIdx.x] : 0;
#pragma unroll
  for (int k = 0; k < SI; ++k) dig[k] = s0 + k * 32 < n ? digit_of(key[k], kmin, shift) : -1;
  __syncthreads();
  int sk[SI];
  {
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < SI; ++k) {
      const unsigned peers = __match_any_sync(FULL, dig[k]);
      const int before = __popc(peers & lt);
      const int base = dig[k] >= 0 ? S.wh[w][dig[k]] : 0;
      __syncwarp();
      if (dig[k] >= 0 && before == 0) S.wh[w][dig[k]] = base + __popc(peers);
      __syncwarp();
      sk[k] = base + before;
    }
  }
  __syncthreads();
  // thread d < 256: digit d's warps' places and its count in the tile, then
  // the tile's exclusive scan over the digits
  {
    int tot = 0;
    if (tid < 256) {
#pragma unroll
      for (int q = 0; q < SW; ++q) {
        const int t = S.wh[q][tid];
        S.wh[q][tid] = tot;
        tot += t;
      }
    }
    int incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) S.wsum[w] = incl;
    __syncthreads();
    if (tid < 256) {
      int pre = 0;
#pragma unroll
      for (int q = 0; q < 256 / 32; ++q) pre += q < w ? S.wsum[q] : 0;
      const int start = pre + incl - tot;
      S.tstart[tid] = start;
      S.gbase[tid] = goff - start;
    }
    __syncthreads();
  }
  int slot[SI];
#pragma unroll
  for (int k = 0; k < SI; ++k) {
    slot[k] = 0;
    if (dig[k] >= 0) {
      slot[k] = S.tstart[dig[k]] + S.wh[w][dig[k]] + sk[k];
      S.sdig[slot[k]] = (unsigned char)dig[k];
      S.stage[slot[k]] = key[k];
    }
  }
  __syncthreads();
  long long val[SI];
#pragma unroll
  for (int k = 0; k < SI; ++k) {
    const long long i = s0 + k * 32;
    val[k] = i < n ? (vin ? vin[i] : i) : 0;
  }
  const int cnt = (int)min((long long)RTILE, n - t0);
#pragma unroll
  for (int t = 0; t < SI; ++t) {
    const int e = t * ST + tid;
    if (e < cnt) kout[S.gbase[S.sdig[e]] + e] = S.stage[e];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SI; ++k)
    if (dig[k] >= 0) S.stage[slot[k]] = val[k];
  __syncthreads();
#pragma unroll
  for (int t = 0; t < SI; ++t) {
    const int e = t * ST + tid;
    if (e < cnt) vout[S.gbase[S.sdig[e]] + e] = S.stage[e];
  }
}

__global__ void k_copy_pairs(const long long* __restrict__ kin, const long long* __restrict__ vin,
                             long long n, long long* __restrict__ kout,
                             long long* __restrict__ vout) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    kout[i] = kin[i];
    vout[i] = vin ? vin[i] : i;
  }
}

unsigned grid_of(long long n, int threads) {
  return (unsigned)std::max<long long>(
      1, std::min<long long>((n + threads - 1) / threads, (long long)sm_count() * 16));
}

// One pinned word pair per host thread and device, for the waits.
int pinned_pair(long long** out) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  thread_local std::map<int, long long*> bufs;
  long long*& p = bufs[dev];
  if (!p) PF_CUDA(cudaHostAlloc((void**)&p, 4 * sizeof(long long), cudaHostAllocDefault));
  *out = p;
  return PF_OK;
}

int read_words(const long long* dev_src, int n, long long* dst, cudaStream_t st) {
  long long* h = nullptr;
  if (int rc = pinned_pair(&h)) return rc;
  PF_CUDA(cudaMemcpyAsync(h, dev_src, sizeof(long long) * n, cudaMemcpyDeviceToHost, st));
  if (int rc = wait_stream(st)) return rc;
  for (int i = 0; i < n; ++i) dst[i] = h[i];
  return PF_OK;
}

struct SortLayout {
  long long* mm;
  long long* hist;
  long long* offs;     // exclusive scan of hist
  long long* scratch;  // scan scratch
  long long* tk;       // ping-pong keys
  long long* tv;       // ping-pong payload
};

SortLayout sort_layout(Arena& a, long long n) {
  SortLayout l{};
  const long long ntiles = std::max<long long>(1, (n + RTILE - 1) / RTILE);
  l.mm = a.take<long long>(4);
  l.hist = a.take<long long>(256 * ntiles);
  l.offs = a.take<long long>(256 * ntiles);
  l.scratch = a.take<long long>(scan_scratch_elems(256 * ntiles));
  l.tk = a.take<long long>(std::max<long long>(n, 1));
  l.tv = a.take<long long>(std::max<long long>(n, 1));
  return l;
}

// The sort itself (workspace laid out by sort_layout).
int sort_pairs(const long long* kin, const long long* vin, long long n, long long* kout,
               long long* vout, const SortLayout& l, cudaStream_t st) {
  if (n == 0) return PF_OK;
  {
    PF_KERNEL("k_minmax", st);
    k_minmax_init<<<1, 1, 0, st>>>(l.mm);
    k_minmax<<<grid_of(n, RT), RT, 0, st>>>(kin, n, l.mm);
  }
  PF_LAUNCH("k_minmax");
  long long mm[2];
  if (int rc = read_words(l.mm, 2, mm, st)) return rc;
  const unsigned long long range = (unsigned long long)mm[1] - (unsigned long long)mm[0];
  const int bits = range ? 64 - __builtin_clzll(range) : 0;
  const int passes = (bits + 7) / 8;
  if (passes == 0) {
    PF_KERNEL("k_copy_pairs", st);
    k_copy_pairs<<<grid_of(n, 256), 256, 0, st>>>(kin, vin, n, kout, vout);
    PF_LAUNCH("k_copy_pairs");
    return PF_OK;
  }
  const int ntiles = (int)((n + RTILE - 1) / RTILE);
  if (int rc = opt_in_smem((const void*)k_rs_scatter, sizeof(ScatterSmem))) return rc;
  const long long* sk = kin;
  const long long* sv = vin;
  for (int p = 0; p < passes; ++p) {
    // the last pass writes the caller's output
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    long long* dk = to_out ? kout : l.tk;
    long long* dv = to_out ? vout : l.tv;
    {
      PF_KERNEL("k_rs_hist", st);
      k_rs_hist<<<ntiles, RT, 0, st>>>(sk, n, mm[0], 8 * p, ntiles, l.hist);
    }
    PF_LAUNCH("k_rs_hist");
    if (int rc = scan_i64(l.hist, l.offs, 256LL * ntiles, false, nullptr, l.scratch, st)) return rc;
    {
      PF_KERNEL("k_rs_scatter", st);
      k_rs_scatter<<<ntiles, ST, sizeof(ScatterSmem), st>>>(sk, sv, n, mm[0], 8 * p, ntiles,
                                                            l.offs, dk, dv);
    }
    PF_LAUNCH("k_rs_scatter");
    sk = dk;
    sv = dv;
  }
  return PF_OK;
}

// ---- unique + reduce ----------------------------------------------------------

enum { OP_SUM = 0, OP_AMAX = 1, OP_AMIN = 2 };
enum { KIND_INT = 0, KIND_FLOAT = 1 };

struct ValCol {
  const void* in;
  void* out;
  int esize, kind, width, op;
};

__global__ void k_heads(const long long* __restrict__ sk, long long n, long long* __restrict__ h) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    h[i] = (i == 0 || sk[i] != sk[i - 1]) ? 1 : 0;
}

// seg (inclusive scan of heads) - 1 is each sorted position's unique index.
__global__ void k_ukeys(const long long* __restrict__ sk, const long long* __restrict__ seg,
                        long long n, long long* __restrict__ ukeys) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (i == 0 || sk[i] != sk[i - 1]) ukeys[seg[i] - 1] = sk[i];
}

// The start value of an op: 0, the lowest value, the highest value.
template <typename T> struct Limits;
template <> struct Limits<long long> {
  __device__ static long long lo() { return LLONG_MIN; }
  __device__ static long long hi() { return LLONG_MAX; }
};
template <> struct Limits<int> {
  __device__ static int lo() { return INT_MIN; }
  __device__ static int hi() { return INT_MAX; }
};
template <> struct Limits<float> {
  __device__ static float lo() { return -__int_as_float(0x7f800000); }
  __device__ static float hi() { return __int_as_float(0x7f800000); }
};
template <> struct Limits<double> {
  __device__ static double lo() { return -__longlong_as_double(0x7ff0000000000000LL); }
  __device__ static double hi() { return __longlong_as_double(0x7ff0000000000000LL); }
};

template <typename T>
__device__ __forceinline__ T identity_of(int op) {
  if (op == OP_SUM) return (T)0;
  if (op == OP_AMAX) return Limits<T>::lo();
  return Limits<T>::hi();
}

template <typename T>
__global__ void k_fill_identity(T* out, long long n, int op) {
  const T v = identity_of<T>(op);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = v;
}

template <typename T>
__device__ __forceinline__ T combine(T a, T b, int op) {
  if (op == OP_SUM) return a + b;
  if (op == OP_AMAX) return a > b ? a : b;
  return a < b ? a : b;
}

// Atomic combine of v into *p.  Integers and float sums use the hardware
// atomics; float max / min use a CAS loop (bounded; *err set if it gives up).
__device__ __forceinline__ void atomic_combine(long long* p, long long v, int op, int*) {
  if (op == OP_SUM) atomicAdd((unsigned long long*)p, (unsigned long long)v);
  else if (op == OP_AMAX) atomicMax(p, v);
  else atomicMin(p, v);
}
__device__ __forceinline__ void atomic_combine(int* p, int v, int op, int*) {
  if (op == OP_SUM) atomicAdd(p, v);
  else if (op == OP_AMAX) atomicMax(p, v);
  else atomicMin(p, v);
}
template <typename F, typename U>
__device__ __forceinline__ void atomic_minmax_float(F* p, F v, int op, int* err) {
  U* pu = reinterpret_cast<U*>(p);
  U old = *pu;
  for (int tries = 0; tries < (1 << 20); ++tries) {
    F cur;
    memcpy(&cur, &old, sizeof(F));
    const F nv = op == OP_AMAX ? (cur > v ? cur : v) : (cur < v ? cur : v);
    if (nv == cur) return;
    U nvu;
    memcpy(&nvu, &nv, sizeof(F));
    const U seen = atomicCAS(pu, old, nvu);
    if (seen == old) return;
    old = seen;
  }
  atomicExch(err, 1);
}
__device__ __forceinline__ void atomic_combine(float* p, float v, int op, int* err) {
  if (op == OP_SUM) atomicAdd(p, v);
  else atomic_minmax_float<float, unsigned>(p, v, op, err);
}
__device__ __forceinline__ void atomic_combine(double* p, double v, int op, int* err) {
  if (op == OP_SUM) atomicAdd(p, v);
  else atomic_minmax_float<double, unsigned long long>(p, v, op, err);
}

// Per sorted position i and element e of the row: the value of row perm[i];
// lanes of one key combine along the warp (sorted positions are adjacent),
// and the warp's first lane of each key does one atomic.
template <typename T>
__global__ void __launch_bounds__(256) k_segreduce(const T* __restrict__ in, T* __restrict__ out,
                                                   int width, int op,
                                                   const long long* __restrict__ perm,
                                                   const long long* __restrict__ seg, long long n,
                                                   int* err) {
  const int lane = threadIdx.x & 31;
  const long long total = n * width;
  for (long long t0 = (long long)blockIdx.x * blockDim.x; t0 < total;
       t0 += (long long)gridDim.x * blockDim.x) {
    // element-major: consecutive threads take consecutive sorted positions
    const long long t = t0 + threadIdx.x;
    const bool live = t < total;
    const int e = live ? (int)(t / n) : 0;
    const long long i = live ? t - (long long)e * n : 0;
    const long long s = live ? seg[i] - 1 : -1;
    T v = live ? in[perm[i] * width + e] : identity_of<T>(op);
    const long long key = live ? s * width + e : -1;
    // segmented inclusive scan down the warp (toward lane 0 as the leader)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_down_sync(FULL, v, o);
      const long long ky = __shfl_down_sync(FULL, key, o);
      // a key's lanes are contiguous, so a lane o above with the same key
      // brings the partial result of [lane + o, lane + 2o) within the key
      if (lane + o < 32 && ky == key) v = combine(v, y, op);
    }
    const long long kup = __shfl_up_sync(FULL, key, 1);
    const bool leader = live && (lane == 0 || kup != key);
    if (leader) atomic_combine(&out[key], v, op, err);
  }
}


// ---- merge of two ascending unique runs ----------------------------------------

constexpr int MAXV = 16;  // value columns

struct VCols {
  const void* a[MAXV];   // run values
  const void* b[MAXV];   // tick values
  void* out[MAXV];
  int kind[MAXV], esize[MAXV], width[MAXV], op[MAXV];
  int n;
};

__device__ __forceinline__ long long lower_bound(const long long* __restrict__ v, long long n,
                                                 long long x) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (v[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// out[dst] = a[i] (combined with b[j] when j >= 0), every element of the row.
template <typename T>
__device__ __forceinline__ void put_row(const VCols& c, int q, long long dst, long long i,
                                        long long j, bool from_b) {
  const int w = c.width[q];
  T* out = reinterpret_cast<T*>(c.out[q]) + dst * w;
  const T* src = reinterpret_cast<const T*>(from_b ? c.b[q] : c.a[q]) + i * w;
  const T* other = reinterpret_cast<const T*>(c.b[q]) + j * w;
  for (int e = 0; e < w; ++e) out[e] = j >= 0 ? combine(src[e], other[e], c.op[q]) : src[e];
}

__device__ __forceinline__ void put_rows(const VCols& c, long long dst, long long i, long long j,
                                         bool from_b) {
  for (int q = 0; q < c.n; ++q) {
    if (c.kind[q] == KIND_FLOAT) {
      if (c.esize[q] == 8) put_row<double>(c, q, dst, i, j, from_b);
      else put_row<float>(c, q, dst, i, j, from_b);
    } else {
      if (c.esize[q] == 8) put_row<long long>(c, q, dst, i, j, from_b);
      else put_row<int>(c, q, dst, i, j, from_b);
    }
  }
}

// Per tick key: its rank in the run and whether the run holds it.
__global__ void k_merge_tick(const long long* __restrict__ run, long long R,
                             const long long* __restrict__ tick, long long T,
                             long long* __restrict__ lb, long long* __restrict__ isnew) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < T;
       k += (long long)gridDim.x * blockDim.x) {
    const long long p = lower_bound(run, R, tick[k]);
    lb[k] = p;
    isnew[k] = (p < R && run[p] == tick[k]) ? 0 : 1;
  }
}

// Every run key moves up by the new tick keys below it; a matched key takes
// the combination of both values.
__global__ void k_merge_place_run(const long long* __restrict__ run, long long R,
                                  const long long* __restrict__ tick, long long T,
                                  const long long* __restrict__ newex,
                                  const long long* __restrict__ new_total, VCols c,
                                  long long* __restrict__ out_keys) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < R;
       j += (long long)gridDim.x * blockDim.x) {
    const long long key = run[j];
    const long long x = lower_bound(tick, T, key);
    const long long below = x < T ? newex[x] : *new_total;
    const long long dst = j + below;
    out_keys[dst] = key;
    put_rows(c, dst, j, (x < T && tick[x] == key) ? x : -1, false);
  }
}

__global__ void k_merge_place_new(const long long* __restrict__ tick, long long T,
                                  const long long* __restrict__ lb,
                                  const long long* __restrict__ isnew,
                                  const long long* __restrict__ newex, VCols c,
                                  long long* __restrict__ out_keys) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < T;
       k += (long long)gridDim.x * blockDim.x) {
    if (!isnew[k]) continue;
    const long long dst = lb[k] + newex[k];
    out_keys[dst] = tick[k];
    put_rows(c, dst, k, -1, true);
  }
}

struct UniqueLayout {
  SortLayout sort;
  long long* sk;
  long long* perm;
  long long* heads;
  long long* seg;
  long long* total;
  long long* scratch;
  int* err;
};

UniqueLayout unique_layout(Arena& a, long long n) {
  UniqueLayout l{};
  l.sort = sort_layout(a, n);
  const long long m = std::max<long long>(n, 1);
  l.sk = a.take<long long>(m);
  l.perm = a.take<long long>(m);
  l.heads = a.take<long long>(m);
  l.seg = a.take<long long>(m);
  l.total = a.take<long long>(1);
  l.scratch = a.take<long long>(scan_scratch_elems(m));
  l.err = a.take<int>(1);
  return l;
}

struct MergeLayout {
  long long* lb;
  long long* isnew;
  long long* newex;
  long long* total;
  long long* scratch;
};

MergeLayout merge_layout(Arena& a, long long T) {
  MergeLayout l{};
  const long long m = std::max<long long>(T, 1);
  l.lb = a.take<long long>(m);
  l.isnew = a.take<long long>(m);
  l.newex = a.take<long long>(m);
  l.total = a.take<long long>(1);
  l.scratch = a.take<long long>(scan_scratch_elems(m));
  return l;
}

int check_cols(int ncols, const int* kinds, const int* esizes, const int* widths, const int* ops,
               const char* what) {
  if (ncols < 0 || ncols > MAXV) return fail(PF_EINVAL, "%s: 0 to %d value columns", what, MAXV);
  for (int q = 0; q < ncols; ++q) {
    if ((kinds[q] != KIND_INT && kinds[q] != KIND_FLOAT) || (esizes[q] != 4 && esizes[q] != 8) ||
        widths[q] < 1 || ops[q] < OP_SUM || ops[q] > OP_AMIN)
      return fail(PF_EINVAL, "%s: value column %d: kind %d, %d bytes, width %d, op %d", what, q,
                  kinds[q], esizes[q], widths[q], ops[q]);
  }
  return PF_OK;
}
}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_sort_pairs_workspace(int64_t n) {
  Arena a(nullptr, 0);
  sort_layout(a, n);
  return a.used + 256;
}

extern "C" int pf_sort_pairs(const int64_t* keys_in, const int64_t* vals_in, int64_t n,
                             int64_t* keys_out, int64_t* vals_out, void* workspace,
                             size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 0 || n > ((int64_t)1 << 40)) return fail(PF_EINVAL, "sort_pairs: bad size");
  if (n > 0 && (!keys_in || !keys_out || !vals_out))
    return fail(PF_EINVAL, "sort_pairs: null pointer");
  Arena a(workspace, workspace_bytes);
  SortLayout l = sort_layout(a, n);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "sort_pairs: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  if (int rc = sort_pairs((const long long*)keys_in, (const long long*)vals_in, n,
                          (long long*)keys_out, (long long*)vals_out, l, st))
    return rc;
  return ok();
}

extern "C" size_t pf_unique_reduce_workspace(int64_t n) {
  Arena a(nullptr, 0);
  unique_layout(a, n);
  return a.used + 256;
}

extern "C" int pf_unique_reduce(const int64_t* keys, int64_t n, int ncols,
                                const void* const* vals_in, void* const* vals_out,
                                const int* kinds, const int* esizes, const int* widths,
                                const int* ops, int64_t* keys_out, int64_t* n_unique,
                                void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 0 || !n_unique) return fail(PF_EINVAL, "unique_reduce: bad arguments");
  if (int rc = check_cols(ncols, kinds, esizes, widths, ops, "unique_reduce")) return rc;
  *n_unique = 0;
  if (n == 0) return ok();
  if (!keys || !keys_out) return fail(PF_EINVAL, "unique_reduce: null keys");
  for (int q = 0; q < ncols; ++q)
    if (!vals_in[q] || !vals_out[q]) return fail(PF_EINVAL, "unique_reduce: null value column");
  Arena a(workspace, workspace_bytes);
  UniqueLayout l = unique_layout(a, n);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "unique_reduce: workspace of %zu bytes, %zu needed",
                workspace_bytes, a.used);
  if (int rc = sort_pairs((const long long*)keys, nullptr, n, l.sk, l.perm, l.sort, st)) return rc;
  {
    PF_KERNEL("k_heads", st);
    k_heads<<<grid_of(n, 256), 256, 0, st>>>(l.sk, n, l.heads);
  }
  PF_LAUNCH("k_heads");
  if (int rc = scan_i64(l.heads, l.seg, n, true, l.total, l.scratch, st)) return rc;
  long long U = 0;
  if (int rc = read_words(l.total, 1, &U, st)) return rc;
  {
    PF_KERNEL("k_ukeys", st);
    k_ukeys<<<grid_of(n, 256), 256, 0, st>>>(l.sk, l.seg, n, (long long*)keys_out);
  }
  PF_LAUNCH("k_ukeys");
  PF_CUDA(cudaMemsetAsync(l.err, 0, sizeof(int), st));
  bool float_minmax = false;
  for (int q = 0; q < ncols; ++q) {
    const long long cells = U * widths[q];
    const long long work = n * widths[q];
    PF_KERNEL("k_segreduce", st);
#define PF_SEG(T)                                                                              \
  k_fill_identity<T><<<grid_of(cells, 256), 256, 0, st>>>((T*)vals_out[q], cells, ops[q]);     \
  k_segreduce<T><<<grid_of(work, 256), 256, 0, st>>>((const T*)vals_in[q], (T*)vals_out[q],    \
                                                     widths[q], ops[q], l.perm, l.seg, n, l.err)
    if (kinds[q] == KIND_FLOAT) {
      float_minmax |= ops[q] != OP_SUM;
      if (esizes[q] == 8) { PF_SEG(double); } else { PF_SEG(float); }
    } else {
      if (esizes[q] == 8) { PF_SEG(long long); } else { PF_SEG(int); }
    }
#undef PF_SEG
  }
  PF_LAUNCH("k_segreduce");
  if (float_minmax) {
    long long e = 0;
    if (int rc = read_words((const long long*)l.err, 1, &e, st)) return rc;
    if ((int)e) return fail(PF_EDEVICE, "unique_reduce: a float max/min gave up");
  }
  *n_unique = U;
  return ok();
}

extern "C" size_t pf_merge_sorted_runs_workspace(int64_t n_tick) {
  Arena a(nullptr, 0);
  merge_layout(a, n_tick);
  return a.used + 256;
}

extern "C" int pf_merge_sorted_runs(const int64_t* run_keys, const void* const* run_vals,
                                    int64_t n_run, const int64_t* tick_keys,
                                    const void* const* tick_vals, int64_t n_tick, int ncols,
                                    const int* kinds, const int* esizes, const int* widths,
                                    const int* ops, int64_t* out_keys, void* const* out_vals,
                                    int64_t* n_out, void* workspace, size_t workspace_bytes,
                                    void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n_run < 0 || n_tick < 0 || !n_out) return fail(PF_EINVAL, "merge_sorted_runs: bad sizes");
  if (int rc = check_cols(ncols, kinds, esizes, widths, ops, "merge_sorted_runs")) return rc;
  if ((n_run > 0 && !run_keys) || (n_tick > 0 && !tick_keys) ||
      (n_run + n_tick > 0 && !out_keys))
    return fail(PF_EINVAL, "merge_sorted_runs: null keys");
  VCols c{};
  c.n = ncols;
  for (int q = 0; q < ncols; ++q) {
    if ((n_run > 0 && !run_vals[q]) || (n_tick > 0 && !tick_vals[q]) || !out_vals[q])
      return fail(PF_EINVAL, "merge_sorted_runs: null value column %d", q);
    c.a[q] = run_vals[q];
    c.b[q] = tick_vals[q];
    c.out[q] = out_vals[q];
    c.kind[q] = kinds[q];
    c.esize[q] = esizes[q];
    c.width[q] = widths[q];
    c.op[q] = ops[q];
  }
  Arena a(workspace, workspace_bytes);
  MergeLayout l = merge_layout(a, n_tick);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "merge_sorted_runs: workspace of %zu bytes, %zu needed",
                workspace_bytes, a.used);
  long long num_new = 0;
  if (n_tick > 0) {
    {
      PF_KERNEL("k_merge_tick", st);
      k_merge_tick<<<grid_of(n_tick, 256), 256, 0, st>>>((const long long*)run_keys, n_run,
                                                         (const long long*)tick_keys, n_tick,
                                                         l.lb, l.isnew);
    }
    PF_LAUNCH("k_merge_tick");
    if (int rc = scan_i64(l.isnew, l.newex, n_tick, false, l.total, l.scratch, st)) return rc;
    if (int rc = read_words(l.total, 1, &num_new, st)) return rc;
  } else {
    PF_CUDA(cudaMemsetAsync(l.total, 0, sizeof(long long), st));
  }
  if (n_run > 0) {
    PF_KERNEL("k_merge_place_run", st);
    k_merge_place_run<<<grid_of(n_run, 256), 256, 0, st>>>(
        (const long long*)run_keys, n_run, (const long long*)tick_keys, n_tick, l.newex, l.total,
        c, (long long*)out_keys);
  }
  PF_LAUNCH("k_merge_place_run");
  if (n_tick > 0) {
    PF_KERNEL("k_merge_place_new", st);
    k_merge_place_new<<<grid_of(n_tick, 256), 256, 0, st>>>((const long long*)tick_keys, n_tick,
                                                            l.lb, l.isnew, l.newex, c,
                                                            (long long*)out_keys);
  }
  PF_LAUNCH("k_merge_place_new");
  *n_out = n_run + num_new;
  return ok();
}
