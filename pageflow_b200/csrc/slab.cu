// The dense slab group-by: sm_100a kernels behind DenseAggregationSlab's add
// and finish (reference operators/aggregation_slab.py:170-246).  A slab is
// direct-addressed over [key_min, key_min + capacity): one occupancy byte and
// one identity-initialised value segment per aggregate.  add folds rows in
// with device atomics (sum / max / min of int64, int32 and float64, the
// operations scatter_reduce_(include_self=True) performs); finish emits the
// occupied keys ascending with their values.
#include "scan.cuh"

namespace pf {
namespace {

constexpr int AT = 256;

__device__ __forceinline__ void fold_f64_max(double* a, double v) {
  unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
  unsigned long long old = *p;
  while (__longlong_as_double((long long)old) < v) {
    const unsigned long long got =
        atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (got == old) break;
    old = got;
  }
}

__device__ __forceinline__ void fold_f64_min(double* a, double v) {
  unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
  unsigned long long old = *p;
  while (__longlong_as_double((long long)old) > v) {
    const unsigned long long got =
        atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (got == old) break;
    old = got;
  }
}

constexpr int MAXV = 8;

struct SlabArgs {
  const void* keys;
  int key_i32;
  long long n, key_min, cap;
  unsigned char* occupied;
  int nvals;
  void* values[MAXV];
  const void* srcs[MAXV];
  int dtype[MAXV], op[MAXV], width[MAXV];
  long long* err;
};

__global__ void __launch_bounds__(AT) k_slab_add(SlabArgs a) {
  for (long long i = (long long)blockIdx.x * AT + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * AT) {
    const long long k = a.key_i32 ? (long long)reinterpret_cast<const int*>(a.keys)[i]
                                   : reinterpret_cast<const long long*>(a.keys)[i];
    const long long off = k - a.key_min;
    if (off < 0 || off >= a.cap) {
      if (a.err) atomicAdd(reinterpret_cast<unsigned long long*>(a.err), 1ULL);
      continue;
    }
    if (!a.occupied[off]) a.occupied[off] = 1;
    for (int v = 0; v < a.nvals; ++v) {
      const int w = a.width[v];
      for (int e = 0; e < w; ++e) {
        const long long d = off * w + e, s = i * w + e;
        switch (a.dtype[v]) {
          case PF_DT_I64: {
            long long* dst = reinterpret_cast<long long*>(a.values[v]) + d;
            const long long x = reinterpret_cast<const long long*>(a.srcs[v])[s];
            if (a.op[v] == PF_AGG_SUM) atomicAdd(reinterpret_cast<unsigned long long*>(dst), (unsigned long long)x);
            else if (a.op[v] == PF_AGG_MAX) atomicMax(dst, x);
            else atomicMin(dst, x);
            break;
          }
          case PF_DT_I32: {
            int* dst = reinterpret_cast<int*>(a.values[v]) + d;
            const int x = reinterpret_cast<const int*>(a.srcs[v])[s];
            if (a.op[v] == PF_AGG_SUM) atomicAdd(dst, x);
            else if (a.op[v] == PF_AGG_MAX) atomicMax(dst, x);
            else atomicMin(dst, x);
            break;
          }
          default: {
            double* dst = reinterpret_cast<double*>(a.values[v]) + d;
            const double x = reinterpret_cast<const double*>(a.srcs[v])[s];
            if (a.op[v] == PF_AGG_SUM) atomicAdd(dst, x);
            else if (a.op[v] == PF_AGG_MAX) fold_f64_max(dst, x);
            else fold_f64_min(dst, x);
            break;
          }
        }
      }
    }
  }
}

// Occupied slots per compaction block.
__global__ void __launch_bounds__(CT) k_occ_count(const unsigned char* __restrict__ occ,
                                                  long long n, long long* __restrict__ bcnt) {
  const long long base = (long long)blockIdx.x * CB;
  int c = 0;
  for (int k = 0; k < CITEMS; ++k) {
    const long long i = base + k * CT + threadIdx.x;
    if (i < n) c += occ[i] != 0;
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

struct FinishArgs {
  const unsigned char* occ;
  long long key_min, cap;
  int nvals;
  const void* values[MAXV];
  void* outs[MAXV];
  int esize[MAXV], width[MAXV];
  long long* keys_out;
  const long long* boff;
};

__global__ void __launch_bounds__(CT) k_occ_emit(FinishArgs a) {
  __shared__ int wsum[CT / 32];
  const long long base = (long long)blockIdx.x * CB + (long long)threadIdx.x * CITEMS;
  bool kp[CITEMS];
  int rank[CITEMS];
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) kp[k] = base + k < a.cap && a.occ[base + k] != 0;
  __shared__ unsigned short rows[CB];
  const int tot = block_compact(kp, rank, rows, wsum);
  const long long o = a.boff[blockIdx.x], b0 = (long long)blockIdx.x * CB;
  for (int e = threadIdx.x; e < tot; e += CT) {
    const long long j = o + e, slot = b0 + rows[e];
    a.keys_out[j] = a.key_min + slot;
    for (int v = 0; v < a.nvals; ++v) {
      const int w = a.width[v];
      if (a.esize[v] == 8) {
        const long long* src = reinterpret_cast<const long long*>(a.values[v]);
        long long* dst = reinterpret_cast<long long*>(a.outs[v]);
        for (int x = 0; x < w; ++x) dst[j * w + x] = src[slot * w + x];
      } else {
        const int* src = reinterpret_cast<const int*>(a.values[v]);
        int* dst = reinterpret_cast<int*>(a.outs[v]);
        for (int x = 0; x < w; ++x) dst[j * w + x] = src[slot * w + x];
      }
    }
  }
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int pf_slab_add(const void* keys, int key_dtype, int64_t n, int64_t key_min,
                           int64_t capacity, uint8_t* occupied, int nvals, void* const* values,
                           const void* const* srcs, const int* dtypes, const int* ops,
                           const int* widths, int64_t* err_count, void* stream) {
  if (nvals < 0 || nvals > MAXV) return fail(PF_EINVAL, "slab_add: at most %d values", MAXV);
  if (key_dtype != PF_DT_I64 && key_dtype != PF_DT_I32)
    return fail(PF_EINVAL, "slab_add: keys must be int64 or int32");
  if (capacity < 0 || n < 0) return fail(PF_EINVAL, "slab_add: negative size");
  if (n == 0) return ok();
  SlabArgs a{};
  a.keys = keys;
  a.key_i32 = key_dtype == PF_DT_I32;
  a.n = n;
  a.key_min = key_min;
  a.cap = capacity;
  a.occupied = occupied;
  a.nvals = nvals;
  for (int v = 0; v < nvals; ++v) {
    if (dtypes[v] != PF_DT_I64 && dtypes[v] != PF_DT_F64 && dtypes[v] != PF_DT_I32)
      return fail(PF_EINVAL, "slab_add: value %d has an unsupported dtype", v);
    if (ops[v] < PF_AGG_SUM || ops[v] > PF_AGG_MIN)
      return fail(PF_EINVAL, "slab_add: value %d has an unsupported op", v);
    if (widths[v] < 1) return fail(PF_EINVAL, "slab_add: value %d has width < 1", v);
    a.values[v] = values[v];
    a.srcs[v] = srcs[v];
    a.dtype[v] = dtypes[v];
    a.op[v] = ops[v];
    a.width[v] = widths[v];
  }
  a.err = (long long*)err_count;
  const long long want = (n + AT - 1) / AT;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(want, sm_count() * 16LL));
  {
    PF_KERNEL("k_slab_add", (cudaStream_t)stream);
    k_slab_add<<<grid, AT, 0, (cudaStream_t)stream>>>(a);
  }
  PF_LAUNCH("k_slab_add");
  return ok();
}

namespace {
struct FinLayout {
  long long* bcnt;
  long long* total;
};
FinLayout fin_layout(Arena& a, int64_t cap) {
  FinLayout l{};
  l.bcnt = a.take<long long>((cap + CB - 1) / CB + 1);
  l.total = a.take<long long>(1);
  return l;
}
}  // namespace

extern "C" size_t pf_slab_finish_workspace(int64_t capacity) {
  Arena a(nullptr, 0);
  fin_layout(a, capacity);
  return a.used + 256;
}

extern "C" int pf_slab_finish(const uint8_t* occupied, int64_t key_min, int64_t capacity,
                              int nvals, const void* const* values, const int* dtypes,
                              const int* widths, int64_t* keys_out, void* const* vals_out,
                              int64_t* host_out, void* workspace, size_t workspace_bytes,
                              void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (nvals < 0 || nvals > MAXV) return fail(PF_EINVAL, "slab_finish: at most %d values", MAXV);
  Arena ar(workspace, workspace_bytes);
  FinLayout l = fin_layout(ar, capacity);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "slab_finish: workspace of %zu bytes, %zu needed", workspace_bytes,
                ar.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  if (capacity == 0) {
    host_out[0] = 0;
    return ok();
  }
  const unsigned nblk = blocks_for(capacity, CB);
  {
    PF_KERNEL("k_occ_count", st);
    k_occ_count<<<nblk, CT, 0, st>>>(occupied, capacity, l.bcnt);
  }
  PF_LAUNCH("k_occ_count");
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.bcnt, nblk, l.total, host_dev);
  }
  PF_LAUNCH("k_scan_counts");
  cudaEvent_t ev;
  if (int rc = record_event(st, &ev)) return rc;
  FinishArgs a{};
  a.occ = occupied;
  a.key_min = key_min;
  a.cap = capacity;
  a.nvals = nvals;
  for (int v = 0; v < nvals; ++v) {
    a.values[v] = values[v];
    a.outs[v] = vals_out[v];
    a.esize[v] = dtypes[v] == PF_DT_I32 ? 4 : 8;
    a.width[v] = widths[v];
  }
  a.keys_out = (long long*)keys_out;
  a.boff = l.bcnt;
  {
    PF_KERNEL("k_occ_emit", st);
    k_occ_emit<<<nblk, CT, 0, st>>>(a);
  }
  PF_LAUNCH("k_occ_emit");
  if (int rc = wait_event(ev)) return rc;
  return ok();
}
