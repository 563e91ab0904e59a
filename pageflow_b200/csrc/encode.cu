// Output-side encoding on the device: partitioned columns written as PFC1
// pages (codec.h) without leaving the GPU, so partitioned intermediates can
// be kept or spilled compressed (the reference compresses its partitioned
// outputs region by region through nvCOMP on the way out:
// IO/codec/region_producer.py, IO/codec/batched_compress.py:27-59).
//
// The pages are byte for byte the ones the host encoder (codec.cu) writes for
// the same values: the same four candidate schemes sized the same way, the
// same choice (the smallest; RAW, FOR, DELTA, RLE in that order on a tie),
// the same block tables, bits and padding.  Two launches and one host wait:
//
//   k_enc_plan    one block a page: per 1024-value mini-block the value and
//                 delta ranges (a block-wide min/max), the run starts (RLE
//                 candidates, at most PFC_RLE_MAX_RUNS runs), every scheme's
//                 size, the choice
//   host          the page sizes back, byte offsets by a prefix sum
//   k_enc_write   one block a page: the header, block tables and bits, each
//                 mini-block's words assembled in shared memory by atomic ORs
//                 and written out whole
#include <algorithm>
#include <vector>

#include "codec.h"
#include "common.cuh"

namespace pf {
namespace {

constexpr int ET = 1024;  // threads of both kernels: one value of a mini-block each
static_assert(ET == PFC_BLOCK, "a thread a mini-block value");

struct PageMeta {
  long long bytes;   // the page's size
  int scheme;
  int rle_vs;        // RLE: the runs' values as FOR or DELTA
  int nruns;
  int pad;
};

__device__ __forceinline__ long long load_value(const unsigned char* col, int esize, long long i) {
  return esize == 8 ? reinterpret_cast<const long long*>(col)[i]
                    : (long long)reinterpret_cast<const int*>(col)[i];
}

__device__ __forceinline__ unsigned bit_width64(unsigned long long r) {
  return r ? 64u - (unsigned)__clzll((long long)r) : 0u;
}

// Block-wide min and max of one value a thread (live threads only).
struct MinMax {
  long long lo, hi;
};
__device__ MinMax block_minmax(long long x, bool live, long long* red) {
  long long lo = live ? x : LLONG_MAX, hi = live ? x : LLONG_MIN;
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(FULL, lo, o));
    hi = max(hi, __shfl_xor_sync(FULL, hi, o));
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    red[w] = lo;
    red[32 + w] = hi;
  }
  __syncthreads();
  if (w == 0) {
    lo = red[lane];
    hi = red[32 + lane];
    for (int o = 16; o; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(FULL, lo, o));
      hi = max(hi, __shfl_xor_sync(FULL, hi, o));
    }
    if (lane == 0) {
      red[0] = lo;
      red[32] = hi;
    }
  }
  __syncthreads();
  return MinMax{red[0], red[32]};
}

// Block-wide exclusive prefix of one flag a thread, and the total.
__device__ int block_prefix(int f, int* wsum, int* total) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(FULL, f);
  const int in_warp = __popc(m & lanemask_lt());
  __syncthreads();
  if (lane == 0) wsum[w] = __popc(m);
  __syncthreads();
  if (w == 0) {
    int x = wsum[lane];
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    wsum[lane] = incl - x;
    if (lane == 31) *total = incl;
  }
  __syncthreads();
  return wsum[w] + in_warp;
}

// One FOR or DELTA mini-block's range over its terms (DELTA: the differences
// after the first value; a block of one value has range 0).
__device__ MinMax block_terms(const long long* v, int cnt, int scheme, long long* red) {
  const int j = threadIdx.x;
  long long t = 0;
  bool live = j < cnt;
  if (live) {
    if (scheme == PFC_DELTA) {
      live = j > 0;
      if (live) t = (long long)((unsigned long long)v[j] - (unsigned long long)v[j - 1]);
    } else {
      t = v[j];
    }
  }
  MinMax m = block_minmax(t, live, red);
  if (m.lo > m.hi) m.lo = m.hi = 0;
  return m;
}

__device__ __forceinline__ long long words_of(unsigned bw, int cnt) {
  return ((long long)bw * cnt + 31) / 32;
}

__device__ __forceinline__ long long align16(long long x) { return (x + 15) / 16 * 16; }

// A stream's bytes from its words: header, block table, words and three
// words of padding, to a 16-byte boundary.
__device__ __forceinline__ long long stream_bytes(long long nblk, long long words) {
  return align16(16 + 32 * nblk + 4 * (words + 3));
}

struct EncShared {
  long long vals[PFC_BLOCK];           // a mini-block's values
  long long rv[PFC_RLE_MAX_RUNS];      // run values
  long long re[PFC_RLE_MAX_RUNS];      // run ends (exclusive rows)
  unsigned words[2 * PFC_BLOCK + 4];   // a mini-block's bits
  long long red[64];
  int wsum[32];
  int total;
  int nruns;
  int over;                            // more runs than an RLE page keeps
};

// The runs of a page's values (while they fit): run values and exclusive
// ends in S.rv / S.re, their number in S.nruns (or S.over).
__device__ void page_runs(const unsigned char* col, int esize, long long p0, long long n,
                          EncShared& S) {
  if (threadIdx.x == 0) {
    S.nruns = 0;
    S.over = 0;
  }
  __syncthreads();
  for (long long b0 = 0; b0 < n; b0 += ET) {
    const long long j = b0 + threadIdx.x;
    int f = 0;
    long long x = 0;
    if (j < n) {
      x = load_value(col, esize, p0 + j);
      f = j == 0 || x != load_value(col, esize, p0 + j - 1);
    }
    const int base = S.nruns;
    const int pos = block_prefix(f, S.wsum, &S.total);
    const int r = base + pos;
    if (f && r < PFC_RLE_MAX_RUNS) {
      S.rv[r] = x;
      if (r > 0) S.re[r - 1] = j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      S.nruns = base + S.total;
      if (S.nruns > PFC_RLE_MAX_RUNS) S.over = 1;
    }
    __syncthreads();
    if (S.over) break;
  }
  if (threadIdx.x == 0 && !S.over && S.nruns > 0) S.re[S.nruns - 1] = n;
  __syncthreads();
}

// A FOR or DELTA stream's bytes over n values read by `get`.
template <typename Get>
__device__ long long stream_size(long long n, int scheme, Get get, EncShared& S) {
  const long long nblk = (n + PFC_BLOCK - 1) / PFC_BLOCK;
  long long words = 0;
  for (long long k = 0; k < nblk; ++k) {
    const int cnt = (int)(n - k * PFC_BLOCK < PFC_BLOCK ? n - k * PFC_BLOCK : PFC_BLOCK);
    if (threadIdx.x < cnt) S.vals[threadIdx.x] = get(k * PFC_BLOCK + threadIdx.x);
    __syncthreads();
    const MinMax m = block_terms(S.vals, cnt, scheme, S.red);
    words += words_of(bit_width64((unsigned long long)m.hi - (unsigned long long)m.lo), cnt);
  }
  return stream_bytes(nblk, words);
}

__global__ void __launch_bounds__(ET) k_enc_plan(const unsigned char* __restrict__ col, int esize,
                                                 const long long* __restrict__ rows, int npages,
                                                 PageMeta* __restrict__ meta) {
  extern __shared__ __align__(16) unsigned char enc_smem[];
  EncShared& S = *reinterpret_cast<EncShared*>(enc_smem);
  for (int p = blockIdx.x; p < npages; p += gridDim.x) {
    const long long p0 = rows[p], n = rows[p + 1] - p0;
    auto value = [&](long long j) { return load_value(col, esize, p0 + j); };
    const long long raw = (long long)esize * n + 16;
    const long long s_for = stream_size(n, PFC_FOR, value, S);
    const long long s_delta = stream_size(n, PFC_DELTA, value, S);
    page_runs(col, esize, p0, n, S);
    long long s_rle = LLONG_MAX;
    int rle_vs = PFC_FOR;
    const int nr = S.nruns;
    if (n > 0 && !S.over) {
      auto rv = [&](long long j) { return S.rv[j]; };
      auto re = [&](long long j) { return S.re[j]; };
      const long long a = stream_size(nr, PFC_FOR, rv, S);
      const long long b = stream_size(nr, PFC_DELTA, rv, S);
      rle_vs = b < a ? PFC_DELTA : PFC_FOR;
      s_rle = min(a, b) + stream_size(nr, PFC_DELTA, re, S);
    }
    int scheme = PFC_RAW;
    long long best = raw;
    if (s_for < best) { best = s_for; scheme = PFC_FOR; }
    if (s_delta < best) { best = s_delta; scheme = PFC_DELTA; }
    if (s_rle < best) { best = s_rle; scheme = PFC_RLE; }
    // the page: 64-byte header, then the chosen streams
    long long bytes = 64;
    if (scheme == PFC_RAW) bytes += align16((long long)esize * n);
    else if (scheme == PFC_RLE) bytes = align16(bytes + s_rle);
    else bytes += best;
    if (threadIdx.x == 0) meta[p] = PageMeta{align16(bytes), scheme, rle_vs, nr, 0};
    __syncthreads();
  }
}

// Writes a FOR or DELTA stream of n values (read by `get`) at `out`;
// returns its bytes.
template <typename Get>
__device__ long long write_stream(unsigned char* out, long long n, int scheme, Get get,
                                  EncShared& S) {
  const long long nblk = (n + PFC_BLOCK - 1) / PFC_BLOCK;
  if (threadIdx.x == 0) {
    PfcStream sh{(uint32_t)scheme, (uint32_t)n, (uint32_t)nblk, 0};
    *reinterpret_cast<PfcStream*>(out) = sh;
  }
  PfcBlock* table = reinterpret_cast<PfcBlock*>(out + 16);
  unsigned* words = reinterpret_cast<unsigned*>(out + 16 + 32 * nblk);
  long long woff = 0;
  for (long long k = 0; k < nblk; ++k) {
    const int cnt = (int)(n - k * PFC_BLOCK < PFC_BLOCK ? n - k * PFC_BLOCK : PFC_BLOCK);
    const int j = threadIdx.x;
    if (j < cnt) S.vals[j] = get(k * PFC_BLOCK + j);
    __syncthreads();
    const MinMax m = block_terms(S.vals, cnt, scheme, S.red);
    const unsigned bw = bit_width64((unsigned long long)m.hi - (unsigned long long)m.lo);
    const long long nw = words_of(bw, cnt);
    for (long long w = j; w < nw + 2; w += ET) S.words[w] = 0;
    __syncthreads();
    if (bw && j < cnt && !(scheme == PFC_DELTA && j == 0)) {
      const long long t = scheme == PFC_DELTA
                              ? (long long)((unsigned long long)S.vals[j] -
                                            (unsigned long long)S.vals[j - 1])
                              : S.vals[j];
      const unsigned long long d = (unsigned long long)t - (unsigned long long)m.lo;
      const unsigned long long bit = (unsigned long long)j * bw;
      unsigned w = (unsigned)(bit >> 5), sh = (unsigned)(bit & 31);
      atomicOr(&S.words[w], (unsigned)(d << sh));
      unsigned done = 32 - sh;
      while (done < bw) {
        ++w;
        atomicOr(&S.words[w], (unsigned)(d >> done));
        done += 32;
      }
    }
    __syncthreads();
    for (long long w = j; w < nw; w += ET) words[woff + w] = S.words[w];
    if (j == 0) {
      PfcBlock b;
      b.base = m.lo;
      b.first = scheme == PFC_DELTA ? S.vals[0] : 0;
      b.word_off = (uint32_t)woff;
      b.bw = bw;
      b.pad[0] = b.pad[1] = 0;
      table[k] = b;
    }
    woff += nw;
    __syncthreads();
  }
  // three zero words, then zeros to the stream's 16-byte end
  const long long end = stream_bytes(nblk, woff);
  for (long long b = 16 + 32 * nblk + 4 * woff + threadIdx.x; b < end; b += ET) out[b] = 0;
  __syncthreads();
  return end;
}

__global__ void __launch_bounds__(ET) k_enc_write(const unsigned char* __restrict__ col,
                                                  int esize, const long long* __restrict__ rows,
                                                  int npages, const PageMeta* __restrict__ meta,
                                                  const long long* __restrict__ offs,
                                                  unsigned char* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char enc_smem[];
  EncShared& S = *reinterpret_cast<EncShared*>(enc_smem);
  for (int p = blockIdx.x; p < npages; p += gridDim.x) {
    const long long p0 = rows[p], n = rows[p + 1] - p0;
    const PageMeta pm = meta[p];
    unsigned char* page = out + offs[p];
    auto value = [&](long long j) { return load_value(col, esize, p0 + j); };
    long long s1 = 0;
    if (pm.scheme == PFC_RAW) {
      const long long nb = (long long)esize * n;
      for (long long i = threadIdx.x; i < n; i += ET) {
        if (esize == 8) reinterpret_cast<long long*>(page + 64)[i] = value(i);
        else reinterpret_cast<int*>(page + 64)[i] = (int)value(i);
      }
      for (long long b = 64 + nb + threadIdx.x; b < pm.bytes; b += ET) page[b] = 0;
    } else if (pm.scheme == PFC_RLE) {
      page_runs(col, esize, p0, n, S);
      auto rv = [&](long long j) { return S.rv[j]; };
      auto re = [&](long long j) { return S.re[j]; };
      const long long nr = pm.nruns;
      s1 = 64 + write_stream(page + 64, nr, pm.rle_vs, rv, S);
      const long long end = s1 + write_stream(page + s1, nr, PFC_DELTA, re, S);
      for (long long b = end + threadIdx.x; b < pm.bytes; b += ET) page[b] = 0;
    } else {
      write_stream(page + 64, n, pm.scheme, value, S);
    }
    if (threadIdx.x == 0) {
      PfcPage h;
      unsigned* hw = reinterpret_cast<unsigned*>(&h);
      for (int i = 0; i < (int)(sizeof(PfcPage) / 4); ++i) hw[i] = 0;
      h.magic = PFC_MAGIC;
      h.scheme = (uint8_t)pm.scheme;
      h.esize = (uint8_t)esize;
      h.n = (uint32_t)n;
      h.nruns = pm.scheme == PFC_RLE ? (uint32_t)pm.nruns : 0u;
      h.s0 = 64;
      h.s1 = pm.scheme == PFC_RLE ? (uint32_t)s1 : 0u;
      h.bytes = (uint32_t)pm.bytes;
      *reinterpret_cast<PfcPage*>(page) = h;
    }
    __syncthreads();
  }
}

struct EncLayout {
  PageMeta* meta;
  long long* rows;
  long long* offs;
};
EncLayout enc_layout(Arena& a, int npages) {
  EncLayout l{};
  l.meta = a.take<PageMeta>((size_t)npages);
  l.rows = a.take<long long>((size_t)npages + 1);
  l.offs = a.take<long long>((size_t)npages + 1);
  return l;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_encode_pages_workspace(int npages) {
  Arena a(nullptr, 0);
  enc_layout(a, std::max(1, npages));
  return a.used + 256;
}

extern "C" int pf_encode_pages(const void* values, int esize, const int64_t* page_rows,
                               int npages, void* out, int64_t capacity, int64_t* page_offsets,
                               void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (esize != 4 && esize != 8) return fail(PF_EINVAL, "encode_pages: esize 4 or 8");
  if (npages < 1 || !page_rows || !page_offsets)
    return fail(PF_EINVAL, "encode_pages: at least one page and its rows");
  for (int p = 0; p < npages; ++p) {
    const long long n = page_rows[p + 1] - page_rows[p];
    if (page_rows[p] < 0 || n < 0 || n > (1LL << 30))
      return fail(PF_EINVAL, "encode_pages: page %d has %lld rows (0 to 2^30)", p, n);
  }
  Arena ar(workspace, workspace_bytes);
  EncLayout l = enc_layout(ar, npages);
  if (!workspace || !ar.fits())
    return fail(PF_ENOSPACE, "encode_pages: workspace of %zu bytes, %zu needed", workspace_bytes,
                ar.used);
  const size_t sm = sizeof(EncShared);
  if (int rc = opt_in_smem((const void*)k_enc_plan, sm)) return rc;
  if (int rc = opt_in_smem((const void*)k_enc_write, sm)) return rc;
  // pageable source: the copy takes the data before it returns
  PF_CUDA(cudaMemcpyAsync(l.rows, page_rows, ((size_t)npages + 1) * sizeof(long long),
                          cudaMemcpyHostToDevice, st));
  const unsigned g = (unsigned)std::min(npages, sm_count() * 2);
  {
    PF_KERNEL("k_enc_plan", st);
    k_enc_plan<<<g, ET, sm, st>>>((const unsigned char*)values, esize, l.rows, npages, l.meta);
  }
  PF_LAUNCH("k_enc_plan");
  std::vector<PageMeta> meta((size_t)npages);
  PF_CUDA(cudaMemcpyAsync(meta.data(), l.meta, meta.size() * sizeof(PageMeta),
                          cudaMemcpyDeviceToHost, st));
  if (int rc = wait_stream(st)) return rc;
  page_offsets[0] = 0;
  for (int p = 0; p < npages; ++p) page_offsets[p + 1] = page_offsets[p] + meta[p].bytes;
  if (page_offsets[npages] > capacity)
    return fail(PF_ENOSPACE, "encode_pages: %lld bytes of pages, capacity %lld",
                (long long)page_offsets[npages], (long long)capacity);
  PF_CUDA(cudaMemcpyAsync(l.offs, page_offsets, ((size_t)npages + 1) * sizeof(long long),
                          cudaMemcpyHostToDevice, st));
  {
    PF_KERNEL("k_enc_write", st);
    k_enc_write<<<g, ET, sm, st>>>((const unsigned char*)values, esize, l.rows, npages, l.meta,
                                   l.offs, (unsigned char*)out);
  }
  PF_LAUNCH("k_enc_write");
  return ok();
}
