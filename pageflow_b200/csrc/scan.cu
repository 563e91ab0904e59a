// int64 scans for the join cores, the slab and the fused path.
#include "scan.cuh"

namespace pf {

__global__ void __launch_bounds__(1024) k_scan_counts(long long* __restrict__ a, long long n,
                                                      long long* total, long long* host) {
  __shared__ long long wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const long long per = (n + 1023) / 1024;
  const long long st = tid * per;
  long long s = 0;
  for (long long q = 0; q < per; ++q) {
    const long long i = st + q;
    if (i < n) s += a[i];
  }
  long long incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
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
    if (lane == 31) {
      if (total) *total = x;
      if (host) *host = x;
    }
  }
  __syncthreads();
  long long ex = wsum[w] + incl - s;
  for (long long q = 0; q < per; ++q) {
    const long long i = st + q;
    if (i < n) {
      const long long t = a[i];
      a[i] = ex;
      ex += t;
    }
  }
}

__global__ void k_copy_i64(const long long* src, long long* dst, long long n) {
  for (long long i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

namespace {

constexpr int ST = 512;
constexpr int SITEMS = 8;
constexpr int SB = ST * SITEMS;  // values a scan block covers

// Block sums of SB values.
__global__ void __launch_bounds__(ST) k_block_sums(const long long* __restrict__ in, long long n,
                                                   long long* __restrict__ sums) {
  const long long base = (long long)blockIdx.x * SB;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SITEMS; ++k) {
    const long long i = base + k * ST + threadIdx.x;
    if (i < n) s += in[i];
  }
  __shared__ long long red[ST / 32];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int q = 0; q < ST / 32; ++q) t += red[q];
    sums[blockIdx.x] = t;
  }
}

// Each block scans its SB values from its offset (thread t: values
// base + t*SITEMS ...).
__global__ void __launch_bounds__(ST) k_block_scan(const long long* __restrict__ in, long long n,
                                                   const long long* __restrict__ offs,
                                                   long long* __restrict__ out, bool inclusive) {
  __shared__ long long wsum[ST / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * SB + (long long)threadIdx.x * SITEMS;
  long long v[SITEMS];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SITEMS; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  long long incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  long long pre = 0;
  for (int q = 0; q < ST / 32; ++q) pre += q < w ? wsum[q] : 0;
  long long r = offs[blockIdx.x] + pre + incl - s;
#pragma unroll
  for (int k = 0; k < SITEMS; ++k) {
    if (inclusive) r += v[k];
    if (base + k < n) out[base + k] = r;
    if (!inclusive) r += v[k];
  }
}

}  // namespace

int64_t scan_scratch_elems(int64_t n) { return (n + SB - 1) / SB + 1; }

int scan_i64(const long long* in, long long* out, long long n, bool inclusive, long long* total,
             long long* scratch, cudaStream_t st) {
  if (n <= 0) {
    if (total) PF_CUDA(cudaMemsetAsync(total, 0, sizeof(long long), st));
    return PF_OK;
  }
  const long long nb = (n + SB - 1) / SB;
  {
    PF_KERNEL("k_block_sums", st);
    k_block_sums<<<(unsigned)nb, ST, 0, st>>>(in, n, scratch);
  }
  PF_LAUNCH("k_block_sums");
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(scratch, nb, total, nullptr);
  }
  PF_LAUNCH("k_scan_counts");
  {
    PF_KERNEL("k_block_scan", st);
    k_block_scan<<<(unsigned)nb, ST, 0, st>>>(in, n, scratch, out, inclusive);
  }
  PF_LAUNCH("k_block_scan");
  return PF_OK;
}

}  // namespace pf
