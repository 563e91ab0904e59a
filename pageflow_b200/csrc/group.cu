// The hash route of the keyed aggregation's pass 1 (PageFlow's
// KeyedAggregate.pass1, operators/aggregate.py:1511-1563):
//
//   pf_group_hash    each row's grouping hash: the key columns' row bytes
//                    read as little-endian int64 words (zero-padded to a
//                    multiple of 8 bytes, _pack_as_int64 :482-505), each word
//                    times its column's coefficient, summed with int64
//                    wrap-around (_hash_key_columns :551-564)
//   pf_hash_buckets  each group hash's bucket among B - the top log2(B) bits of
//                    its mix64 (_bucket_ids :107-116) - and the groups per
//                    bucket
// The grouping itself (unique hashes ascending, one key representative and
// the partials per group) is pf_unique_reduce over the hashes.
#include <algorithm>

#include "common.cuh"

namespace pf {
namespace {

constexpr int HMAXC = 8;
constexpr int HT = 256;

struct HashCols {
  const unsigned char* col[HMAXC];
  const long long* coeff[HMAXC];
  int rb[HMAXC];     // row bytes
  int words[HMAXC];  // int64 words a row (rb rounded up to 8)
  int path[HMAXC];   // 0: whole aligned words, 1: one aligned 4-byte row, 2: bytes
  int n;
};

__device__ __forceinline__ unsigned long long load_word(const HashCols& h, int c,
                                                        const unsigned char* row, int w) {
  if (h.path[c] == 0) return reinterpret_cast<const unsigned long long*>(row)[w];
  if (h.path[c] == 1) return (unsigned long long)*reinterpret_cast<const unsigned*>(row);
  unsigned long long v = 0;
  const int b0 = 8 * w, b1 = min(h.rb[c], b0 + 8);
  for (int b = b0; b < b1; ++b) v |= (unsigned long long)row[b] << (8 * (b - b0));
  return v;
}

__global__ void __launch_bounds__(HT) k_group_hash(HashCols h, long long n,
                                                   long long* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * HT + threadIdx.x; i < n;
       i += (long long)gridDim.x * HT) {
    unsigned long long acc = 0;
    for (int c = 0; c < h.n; ++c) {
      const unsigned char* row = h.col[c] + i * h.rb[c];
      for (int w = 0; w < h.words[c]; ++w)
        acc += load_word(h, c, row, w) * (unsigned long long)h.coeff[c][w];
    }
    out[i] = (long long)acc;
  }
}

__global__ void __launch_bounds__(HT) k_hash_buckets(const long long* __restrict__ hash,
                                                     long long n, int logB,
                                                     int* __restrict__ bucket,
                                                     long long* __restrict__ counts) {
  extern __shared__ int hc[];
  const int B = 1 << logB;
  for (int b = threadIdx.x; b < B; b += HT) hc[b] = 0;
  __syncthreads();
  for (long long i = (long long)blockIdx.x * HT + threadIdx.x; i < n;
       i += (long long)gridDim.x * HT) {
    const int b = logB ? bucket_of_hash(mix64((uint64_t)hash[i]), logB) : 0;
    bucket[i] = b;
    atomicAdd(&hc[b], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < B; b += HT)
    if (hc[b]) atomicAdd((unsigned long long*)&counts[b], (unsigned long long)hc[b]);
}

unsigned grid_for_rows(long long n) {
  return (unsigned)std::max<long long>(
      1, std::min<long long>((n + HT - 1) / HT, (long long)sm_count() * 16));
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int pf_group_hash(const void* const* key_cols, const int* row_bytes,
                             const int64_t* const* coeffs, int ncols, int64_t n, int64_t* hash_out,
                             void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ncols < 1 || ncols > HMAXC) return fail(PF_EINVAL, "group_hash: 1 to %d key columns", HMAXC);
  if (n < 0) return fail(PF_EINVAL, "group_hash: negative rows");
  HashCols h{};
  h.n = ncols;
  for (int c = 0; c < ncols; ++c) {
    if (row_bytes[c] < 1) return fail(PF_EINVAL, "group_hash: key column %d has no bytes", c);
    if (n > 0 && (!key_cols[c] || !coeffs[c]))
      return fail(PF_EINVAL, "group_hash: key column %d is null", c);
    h.col[c] = (const unsigned char*)key_cols[c];
    h.coeff[c] = (const long long*)coeffs[c];
    h.rb[c] = row_bytes[c];
    h.words[c] = (row_bytes[c] + 7) / 8;
    const uintptr_t a = (uintptr_t)key_cols[c];
    h.path[c] = (row_bytes[c] % 8 == 0 && a % 8 == 0) ? 0
                : (row_bytes[c] == 4 && a % 4 == 0)   ? 1
                                                      : 2;
  }
  if (n == 0) return ok();
  if (!hash_out) return fail(PF_EINVAL, "group_hash: null output");
  {
    PF_KERNEL("k_group_hash", st);
    k_group_hash<<<grid_for_rows(n), HT, 0, st>>>(h, n, (long long*)hash_out);
  }
  PF_LAUNCH("k_group_hash");
  return ok();
}

extern "C" int pf_hash_buckets(const int64_t* hash, int64_t n, int B, int32_t* bucket_out,
                               int64_t* counts_out, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (B < 1 || B > 4096 || (B & (B - 1)))
    return fail(PF_EINVAL, "hash_buckets: B must be a power of two <= 4096");
  if (n < 0 || !counts_out) return fail(PF_EINVAL, "hash_buckets: bad arguments");
  PF_CUDA(cudaMemsetAsync(counts_out, 0, sizeof(int64_t) * B, st));
  if (n == 0) return ok();
  if (!hash || !bucket_out) return fail(PF_EINVAL, "hash_buckets: null pointer");
  {
    PF_KERNEL("k_hash_buckets", st);
    k_hash_buckets<<<grid_for_rows(n), HT, sizeof(int) * B, st>>>(
        (const long long*)hash, n, log2_exact((uint64_t)B), bucket_out, (long long*)counts_out);
  }
  PF_LAUNCH("k_hash_buckets");
  return ok();
}
