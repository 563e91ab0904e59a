// Late materialization after a join: the rows of several columns at one
// index array, in one launch (the reference gathers each output column with
// its own torch.index_select / index_with_null: operators/hashjoin.py:
// 355-377, conversion.py:39-50).
//
// Output row i of column c is input row idx[i] of column c, or, where
// idx[i] is the null sentinel and nulls are allowed, a row whose every
// element is the column's null element.  An index outside [0, n_src) (and
// not an allowed null) writes the null row too and is counted in bad[0], so
// the kernel never reads out of bounds.  A thread copies one output row of
// every column (the index read once), in the widest steps (16 bytes down to
// 1) that the row width and the columns' alignment allow; where every row is
// one such step, a thread takes several rows with all their loads issued
// before the first store.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace pf {
namespace {

constexpr int GT = 256;
constexpr int GMAXC = 16;

struct GatherArgs {
  const unsigned char* in[GMAXC];
  unsigned char* out[GMAXC];
  int row_bytes[GMAXC];
  unsigned long long null_elem[GMAXC];  // the null element's bit pattern
  int esize[GMAXC];
  int wsize[GMAXC];  // bytes a copy step: the widest of 16, 8, 4, 2, 1 that
                     // divides the row and both base addresses
  const long long* idx;
  long long n, n_src;
  long long null_idx;
  int allow_null;
  int ncols;
  unsigned long long* bad;
};

// Source reads through the read-only path (the columns do not change during
// the launch).
template <typename W>
__device__ __forceinline__ W ldg_word(const W* p) { return __ldg(p); }
template <>
__device__ __forceinline__ uint4 ldg_word<uint4>(const uint4* p) { return __ldg(p); }

template <typename W>
__device__ __forceinline__ void copy_row(const GatherArgs& a, int c, long long i, long long j,
                                         bool null_row) {
  const int words = a.row_bytes[c] / (int)sizeof(W);
  W* dst = reinterpret_cast<W*>(a.out[c] + i * a.row_bytes[c]);
  if (!null_row) {
    const W* src = reinterpret_cast<const W*>(a.in[c] + j * a.row_bytes[c]);
    for (int w = 0; w < words; ++w) dst[w] = ldg_word(src + w);
    return;
  }
  // the null row: the element's bytes repeated along the row
  for (int w = 0; w < words; ++w) {
    W pat;
    unsigned char* pb = reinterpret_cast<unsigned char*>(&pat);
    for (int b = 0; b < (int)sizeof(W); ++b)
      pb[b] = (unsigned char)(a.null_elem[c] >> (8 * ((w * (int)sizeof(W) + b) % a.esize[c])));
    dst[w] = pat;
  }
}

template <int NC>
__global__ void __launch_bounds__(GT) k_gather(GatherArgs a) {
  // a thread takes one output row of every column: the index is read once
  // and the columns' loads are in flight together
  const int ncols = NC > 0 ? NC : a.ncols;
  unsigned long long bad = 0;
  for (long long i = (long long)blockIdx.x * GT + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * GT) {
    const long long j = a.idx[i];
    bool null_row = false;
    if (a.allow_null && j == a.null_idx) {
      null_row = true;
    } else if (j < 0 || j >= a.n_src) {
      null_row = true;
      ++bad;
    }
#pragma unroll
    for (int c = 0; c < (NC > 0 ? NC : GMAXC); ++c) {
      if (NC == 0 && c >= ncols) break;
      switch (a.wsize[c]) {
        case 16: copy_row<uint4>(a, c, i, j, null_row); break;
        case 8: copy_row<unsigned long long>(a, c, i, j, null_row); break;
        case 4: copy_row<unsigned>(a, c, i, j, null_row); break;
        case 2: copy_row<unsigned short>(a, c, i, j, null_row); break;
        default: copy_row<unsigned char>(a, c, i, j, null_row); break;
      }
    }
  }
  for (int o = 16; o; o >>= 1) bad += __shfl_xor_sync(FULL, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(a.bad, bad);
}

#ifndef PF_GATHER_LDG
#define PF_GATHER_LDG 1
#endif
#ifndef PF_GATHER_R
#define PF_GATHER_R 4
#endif
constexpr int GR = PF_GATHER_R;  // rows a thread takes together

template <typename W>
__device__ __forceinline__ W load_word(const unsigned char* base, long long j) {
  const W* p = reinterpret_cast<const W*>(base) + j;
  return PF_GATHER_LDG ? ldg_word(p) : *p;
}

// One word a row in every column (row_bytes == wsize): GR rows a thread, the
// indexes and then every column's words loaded before the first store.
template <int NC>
__global__ void __launch_bounds__(GT) k_gather_words(GatherArgs a) {
  unsigned long long bad = 0;
  for (long long b = (long long)blockIdx.x * GT * GR; b < a.n;
       b += (long long)gridDim.x * GT * GR) {
    long long j[GR];
    bool null_row[GR];
#pragma unroll
    for (int r = 0; r < GR; ++r) {
      const long long i = b + r * GT + threadIdx.x;
      j[r] = i < a.n ? a.idx[i] : 0;
    }
#pragma unroll
    for (int r = 0; r < GR; ++r) {
      const bool live = b + r * GT + threadIdx.x < a.n;
      null_row[r] = false;
      if (live && a.allow_null && j[r] == a.null_idx) {
        null_row[r] = true;
      } else if (live && (j[r] < 0 || j[r] >= a.n_src)) {
        null_row[r] = true;
        ++bad;
      }
      if (!live) null_row[r] = true;
    }
    uint4 v[NC][GR];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int r = 0; r < GR; ++r) {
        if (null_row[r]) continue;
        switch (a.wsize[c]) {
          case 16: v[c][r] = load_word<uint4>(a.in[c], j[r]); break;
          case 8: {
            const unsigned long long x = load_word<unsigned long long>(a.in[c], j[r]);
            v[c][r].x = (unsigned)x;
            v[c][r].y = (unsigned)(x >> 32);
            break;
          }
          case 4: v[c][r].x = load_word<unsigned>(a.in[c], j[r]); break;
          case 2: v[c][r].x = load_word<unsigned short>(a.in[c], j[r]); break;
          default: v[c][r].x = load_word<unsigned char>(a.in[c], j[r]); break;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int r = 0; r < GR; ++r) {
        const long long i = b + r * GT + threadIdx.x;
        if (i >= a.n) continue;
        if (null_row[r]) {
          copy_row<unsigned char>(a, c, i, 0, true);
          continue;
        }
        unsigned char* out = a.out[c];
        switch (a.wsize[c]) {
          case 16: reinterpret_cast<uint4*>(out)[i] = v[c][r]; break;
          case 8:
            reinterpret_cast<unsigned long long*>(out)[i] =
                ((unsigned long long)v[c][r].y << 32) | v[c][r].x;
            break;
          case 4: reinterpret_cast<unsigned*>(out)[i] = v[c][r].x; break;
          case 2: reinterpret_cast<unsigned short*>(out)[i] = (unsigned short)v[c][r].x; break;
          default: out[i] = (unsigned char)v[c][r].x; break;
        }
      }
    }
  }
  for (int o = 16; o; o >>= 1) bad += __shfl_xor_sync(FULL, bad, o);
  if ((threadIdx.x & 31) == 0 && bad && a.bad) atomicAdd(a.bad, bad);
}


// ---- zero copy: rows read in place from pinned host segments ----------------
//
// A column spread over host segments (segment s holds rows [seg_rows[s],
// seg_rows[s + 1]) at seg[c * nseg + s], device aliases of pinned host
// memory).  Output row i of column c is row idx[i] - base of the column read
// over the host link; a null index gives the null row, an index outside the
// segments the null row too, counted in bad[0] (never read).  With order,
// thread k takes output row order[k], so that consecutive threads read
// consecutive host rows when order sorts the indexes.
constexpr int ZT = 256;
constexpr int ZMAXSEG = 1024;  // segments the block's shared-memory table holds

struct SegGatherArgs {
  const unsigned char* const* seg;  // [ncols * nseg]
  const long long* seg_rows;        // [nseg + 1] ascending
  int nseg, ncols;
  long long base;
  const long long* idx;
  const long long* order;           // or null
  long long n;
  long long null_idx;
  int allow_null;
  int row_bytes[GMAXC];
  int esize[GMAXC];
  unsigned long long null_elem[GMAXC];
  unsigned char* out[GMAXC];
  unsigned long long* bad;
};

__global__ void __launch_bounds__(ZT) k_gather_segments(SegGatherArgs a) {
  __shared__ long long bounds[ZMAXSEG + 1];
  for (int s = threadIdx.x; s <= a.nseg; s += ZT) bounds[s] = a.seg_rows[s];
  __syncthreads();
  unsigned long long bad = 0;
  for (long long k = (long long)blockIdx.x * ZT + threadIdx.x; k < a.n;
       k += (long long)gridDim.x * ZT) {
    const long long i = a.order ? a.order[k] : k;
    const long long j = a.idx[i];
    int seg = -1;
    long long row = 0;
    if (!(a.allow_null && j == a.null_idx)) {
      const long long r = j + a.base;
      if (r >= bounds[0] && r < bounds[a.nseg]) {
        int lo = 0, hi = a.nseg;  // bounds[lo] <= r < bounds[hi]
        while (hi - lo > 1) {
          const int m = (lo + hi) >> 1;
          if (bounds[m] <= r) lo = m;
          else hi = m;
        }
        seg = lo;
        row = r - bounds[lo];
      } else {
        ++bad;
      }
    }
    for (int c = 0; c < a.ncols; ++c) {
      const int rb = a.row_bytes[c];
      unsigned char* dst = a.out[c] + i * rb;
      if (seg >= 0) {
        const unsigned char* src = a.seg[(long long)c * a.nseg + seg] + row * rb;
        for (int b = 0; b < rb; ++b) dst[b] = src[b];
      } else {
        for (int b = 0; b < rb; ++b)
          dst[b] = (unsigned char)(a.null_elem[c] >> (8 * (b % a.esize[c])));
      }
    }
  }
  for (int o = 16; o; o >>= 1) bad += __shfl_xor_sync(FULL, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(a.bad, bad);
}
}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int pf_gather(const void* const* cols_in, void* const* cols_out, const int* row_bytes,
                         const int* elem_bytes, const uint64_t* null_elem, int ncols,
                         const int64_t* idx, int64_t n, int64_t n_src, int allow_null,
                         int64_t null_idx, int64_t* bad, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ncols < 1 || ncols > GMAXC) return fail(PF_EINVAL, "gather: 1 to %d columns", GMAXC);
  if (n < 0 || n_src < 0) return fail(PF_EINVAL, "gather: negative sizes");
  if (!bad) return fail(PF_EINVAL, "gather: null bad counter");
  GatherArgs a{};
  for (int c = 0; c < ncols; ++c) {
    const int e = elem_bytes[c];
    if (row_bytes[c] < 1 || (e != 1 && e != 2 && e != 4 && e != 8) || row_bytes[c] % e)
      return fail(PF_EINVAL, "gather: column %d: %d-byte rows of %d-byte elements", c,
                  row_bytes[c], e);
    if ((n > 0 && !cols_out[c]) || (n_src > 0 && !cols_in[c]))
      return fail(PF_EINVAL, "gather: column %d is null", c);
    a.in[c] = (const unsigned char*)cols_in[c];
    a.out[c] = (unsigned char*)cols_out[c];
    a.row_bytes[c] = row_bytes[c];
    a.esize[c] = e;
    a.null_elem[c] = null_elem ? null_elem[c] : 0ULL;
    int w = 16;
    while (w > 1 && (row_bytes[c] % w || (uintptr_t)cols_in[c] % w || (uintptr_t)cols_out[c] % w))
      w >>= 1;
    a.wsize[c] = w;
  }
  if (n == 0) return ok();
  if (!idx) return fail(PF_EINVAL, "gather: null index");
  a.idx = (const long long*)idx;
  a.n = n;
  a.n_src = n_src;
  a.null_idx = null_idx;
  a.allow_null = allow_null;
  a.ncols = ncols;
  a.bad = (unsigned long long*)bad;
  const unsigned gx = (unsigned)std::max<long long>(
      1, std::min<long long>((n + GT - 1) / GT, (long long)sm_count() * 8));
  bool words = ncols <= 4;
  for (int c = 0; c < ncols; ++c) words = words && a.row_bytes[c] == a.wsize[c];
  if (words) {
    const unsigned gw = (unsigned)std::max<long long>(
        1, std::min<long long>((n + GT * GR - 1) / (GT * GR), (long long)sm_count() * 8));
#ifndef PF_GATHER_SPLIT
#define PF_GATHER_SPLIT 1
#endif
    if (PF_GATHER_SPLIT) {
      // a pass a column: one column's random reads at a time (2 int64
      // columns at 100M random rows: 4.70 ms, both columns in one pass with
      // 2 rows a thread 4.76, with 4 rows a thread 5.14)
      for (int c = 0; c < ncols; ++c) {
        GatherArgs one = a;
        one.ncols = 1;
        one.in[0] = a.in[c];
        one.out[0] = a.out[c];
        one.row_bytes[0] = a.row_bytes[c];
        one.null_elem[0] = a.null_elem[c];
        one.esize[0] = a.esize[c];
        one.wsize[0] = a.wsize[c];
        if (c > 0) one.bad = nullptr;
        PF_KERNEL("k_gather_words", st);
        k_gather_words<1><<<gw, GT, 0, st>>>(one);
      }
      PF_LAUNCH("k_gather_words");
      return ok();
    }
    PF_KERNEL("k_gather_words", st);
    switch (ncols) {
      case 1: k_gather_words<1><<<gw, GT, 0, st>>>(a); break;
      case 2: k_gather_words<2><<<gw, GT, 0, st>>>(a); break;
      case 3: k_gather_words<3><<<gw, GT, 0, st>>>(a); break;
      default: k_gather_words<4><<<gw, GT, 0, st>>>(a); break;
    }
    PF_LAUNCH("k_gather_words");
    return ok();
  }
  {
    PF_KERNEL("k_gather", st);
    switch (ncols) {
      case 1: k_gather<1><<<gx, GT, 0, st>>>(a); break;
      case 2: k_gather<2><<<gx, GT, 0, st>>>(a); break;
      case 3: k_gather<3><<<gx, GT, 0, st>>>(a); break;
      case 4: k_gather<4><<<gx, GT, 0, st>>>(a); break;
      default: k_gather<0><<<gx, GT, 0, st>>>(a); break;
    }
  }
  PF_LAUNCH("k_gather");
  return ok();
}

extern "C" size_t pf_gather_segments_workspace(int ncols, int nseg) {
  Arena a(nullptr, 0);
  a.take<const unsigned char*>((size_t)ncols * nseg);
  a.take<long long>((size_t)nseg + 1);
  return a.used + 256;
}

extern "C" int pf_gather_segments(void* const* seg_ptrs, const int64_t* seg_rows, int nseg,
                                  int64_t base, int ncols, const int* row_bytes,
                                  const int* elem_bytes, const uint64_t* null_elem,
                                  const int64_t* idx, const int64_t* order, int64_t n,
                                  int allow_null, int64_t null_idx, void* const* cols_out,
                                  int64_t* bad, void* workspace, size_t workspace_bytes,
                                  void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ncols < 1 || ncols > GMAXC) return fail(PF_EINVAL, "gather_segments: 1 to %d columns", GMAXC);
  if (nseg < 1 || nseg > ZMAXSEG)
    return fail(PF_EINVAL, "gather_segments: 1 to %d segments, got %d", ZMAXSEG, nseg);
  if (n < 0) return fail(PF_EINVAL, "gather_segments: negative rows");
  if (!bad || !seg_ptrs || !seg_rows) return fail(PF_EINVAL, "gather_segments: null argument");
  for (int s = 0; s < nseg; ++s)
    if (seg_rows[s + 1] < seg_rows[s])
      return fail(PF_EINVAL, "gather_segments: segment rows must ascend");
  Arena ar(workspace, workspace_bytes);
  const unsigned char** dseg = ar.take<const unsigned char*>((size_t)ncols * nseg);
  long long* drows = ar.take<long long>((size_t)nseg + 1);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "gather_segments: workspace of %zu bytes, %zu needed",
                workspace_bytes, ar.used);
  SegGatherArgs a{};
  for (int c = 0; c < ncols; ++c) {
    const int e = elem_bytes[c];
    if (row_bytes[c] < 1 || (e != 1 && e != 2 && e != 4 && e != 8) || row_bytes[c] % e)
      return fail(PF_EINVAL, "gather_segments: column %d: %d-byte rows of %d-byte elements", c,
                  row_bytes[c], e);
    if (n > 0 && !cols_out[c]) return fail(PF_EINVAL, "gather_segments: column %d is null", c);
    a.row_bytes[c] = row_bytes[c];
    a.esize[c] = e;
    a.null_elem[c] = null_elem ? null_elem[c] : 0ULL;
    a.out[c] = (unsigned char*)cols_out[c];
  }
  // each segment's device alias (pinned host memory: the rows stay where they are)
  std::vector<const unsigned char*> alias((size_t)ncols * nseg);
  for (size_t k = 0; k < alias.size(); ++k) {
    void* d = nullptr;
    if (seg_rows[k % nseg + 1] > seg_rows[k % nseg]) {
      if (!seg_ptrs[k]) return fail(PF_EINVAL, "gather_segments: a segment with rows is null");
      cudaError_t e = cudaHostGetDevicePointer(&d, seg_ptrs[k], 0);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PF_EINVAL, "gather_segments: a segment is not pinned host memory (%s)",
                    cudaGetErrorString(e));
      }
    }
    alias[k] = (const unsigned char*)d;
  }
  if (n == 0) return ok();
  if (!idx) return fail(PF_EINVAL, "gather_segments: null index");
  // pageable sources: the copies take the data before they return
  PF_CUDA(cudaMemcpyAsync(dseg, alias.data(), alias.size() * sizeof(void*),
                          cudaMemcpyHostToDevice, st));
  PF_CUDA(cudaMemcpyAsync(drows, seg_rows, ((size_t)nseg + 1) * sizeof(long long),
                          cudaMemcpyHostToDevice, st));
  a.seg = dseg;
  a.seg_rows = drows;
  a.nseg = nseg;
  a.ncols = ncols;
  a.base = base;
  a.idx = (const long long*)idx;
  a.order = (const long long*)order;
  a.n = n;
  a.null_idx = null_idx;
  a.allow_null = allow_null;
  a.bad = (unsigned long long*)bad;
  const unsigned g = (unsigned)std::max<long long>(
      1, std::min<long long>((n + ZT - 1) / ZT, (long long)sm_count() * 8));
  {
    PF_KERNEL("k_gather_segments", st);
    k_gather_segments<<<g, ZT, 0, st>>>(a);
  }
  PF_LAUNCH("k_gather_segments");
  return ok();
}
