// Shared pieces of the pageflow_b200 kernels: the key hash, error reporting
// through the C ABI, the bump allocator over a caller's workspace, and the
// bounded host wait.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/pageflow_b200.h"

namespace pf {

constexpr unsigned FULL = 0xffffffffu;

// Murmur3's 64-bit finalizer.  A join key's radix bucket is the top log2(B)
// bits of mix64(key), the function PageFlow partitions by
// (operators/kernels/kernel_utils.cuh:18-22, operators/aggregate.py:95-116),
// so both sides of a join, and the reference's own buckets, agree bit for bit.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// The bucket among 2^logB of a key's hash: its top logB bits.
__host__ __device__ __forceinline__ int bucket_of_hash(uint64_t h, int logB) {
  return logB ? (int)(h >> (64 - logB)) : 0;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

// ---- errors ---------------------------------------------------------------

// Records a failure message for pf_last_error() and returns `code`.
int fail(int code, const char* fmt, ...);
// Clears the calling thread's message; returns PF_OK.
int ok();
// PF_ECUDA with the CUDA error string when `e` is an error, else PF_OK.
int cuda_status(cudaError_t e, const char* what);

#define PF_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::pf::cuda_status(e_, #call); \
  } while (0)

#define PF_LAUNCH(what)                                         \
  do {                                                          \
    cudaError_t e_ = cudaGetLastError();                        \
    if (e_ != cudaSuccess) return ::pf::cuda_status(e_, what);  \
  } while (0)

// ---- workspace --------------------------------------------------------------

// A bump allocator over the caller's workspace.  With base == nullptr it
// only sums the sizes, so one layout function serves both *_workspace() and
// the call itself.
struct Arena {
  char* base;
  size_t cap;
  size_t used = 0;
  Arena(void* b, size_t c) : base((char*)b), cap(c) {}
  template <typename T>
  T* take(size_t count, size_t align = 256) {
    used = (used + align - 1) / align * align;
    T* p = base ? (T*)(base + used) : nullptr;
    used += count * sizeof(T);
    return p;
  }
  // the caller's workspace starts on a 256-byte boundary (as cudaMalloc and
  // torch's allocator return): every carved buffer is then aligned for the
  // 16-byte vector accesses and bulk copies the kernels make
  bool aligned() const { return ((uintptr_t)base & 255) == 0; }
  bool fits() const { return aligned() && used <= cap; }
};

// ---- host side helpers --------------------------------------------------------

// The SM count of the current device (cached per device).
int sm_count();
// The device alias of pinned host memory; PF_EINVAL when `host` is not pinned.
int host_alias(void* host, void** dev);
// Records an event on `st` and waits for it with a bounded poll
// (pf_set_wait_timeout_ms); one event per (device, stream, host thread).
int wait_stream(cudaStream_t st);
// The same in two halves, so that work queued in between overlaps the wait:
// record_event marks the point, wait_event polls for it.
int record_event(cudaStream_t st, cudaEvent_t* ev);
int wait_event(cudaEvent_t ev);
// Launch accounting: every kernel launch of the library sits inside a
// LaunchScope, which counts it (pf_launch_count) and, while the calling
// thread profiles (pf_profile_begin / pf_profile_end), brackets it with a
// pair of CUDA events on its stream.
void launch_begin(const char* name, cudaStream_t st);
void launch_end(cudaStream_t st);
struct LaunchScope {
  cudaStream_t st;
  LaunchScope(const char* name, cudaStream_t s) : st(s) { launch_begin(name, s); }
  ~LaunchScope() { launch_end(st); }
};
#define PF_KERNEL(name, st) ::pf::LaunchScope pf_launch_scope_(name, st)

// Raises a kernel's dynamic shared memory limit to `bytes` (past the default
// 48 KiB), once per (kernel, device) at the largest size asked for so far.
int opt_in_smem(const void* fn, size_t bytes);
// The smallest power of two >= x (x >= 1).
inline uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}
inline int log2_exact(uint64_t p) {
  int l = 0;
  while ((1ULL << l) < p) ++l;
  return l;
}
inline unsigned blocks_for(int64_t n, int per) {
  int64_t b = (n + per - 1) / per;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace pf
