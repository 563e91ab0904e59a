// A counting device allocator for torch's CUDAPluggableAllocator (test
// infrastructure): every block it hands out is recorded, so a test can check
// that a library's device buffers all came through the installed allocator,
// as PageFlow's pooled arena is installed (main.py:1389-1395).
#include <cuda_runtime.h>
#include <sys/types.h>

#include <map>
#include <mutex>

namespace {
std::mutex mu;
std::map<char*, size_t> live;
size_t served_bytes = 0, served_blocks = 0;
}  // namespace

extern "C" {
void* pf_test_alloc(ssize_t size, int device, cudaStream_t) {
  void* p = nullptr;
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  const cudaError_t rc = cudaMalloc(&p, size > 0 ? (size_t)size : 1);
  if (cur != device) cudaSetDevice(cur);
  if (rc != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  live[(char*)p] = (size_t)size;
  served_bytes += (size_t)size;
  ++served_blocks;
  return p;
}

void pf_test_free(void* ptr, ssize_t, int, cudaStream_t) {
  {
    std::lock_guard<std::mutex> g(mu);
    live.erase((char*)ptr);
  }
  cudaFree(ptr);
}

size_t pf_test_live_bytes() {
  std::lock_guard<std::mutex> g(mu);
  size_t t = 0;
  for (auto& kv : live) t += kv.second;
  return t;
}

size_t pf_test_served_blocks() {
  std::lock_guard<std::mutex> g(mu);
  return served_blocks;
}

// 1 when [p, p + n) lies inside one live block
int pf_test_owns(const void* p, size_t n) {
  std::lock_guard<std::mutex> g(mu);
  auto it = live.upper_bound((char*)p);
  if (it == live.begin()) return 0;
  --it;
  return (const char*)p >= it->first && (const char*)p + n <= it->first + it->second;
}
}
