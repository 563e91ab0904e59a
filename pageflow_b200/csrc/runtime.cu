// Host-side runtime of the C ABI: error messages, the bounded host wait, and
// device attributes.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <thread>
#include <utility>
#include <string>
#include <vector>
#include <algorithm>

#include "common.cuh"

namespace pf {

namespace {
thread_local char g_msg[1024] = "";
std::atomic<int64_t> g_wait_ms{120000};
}  // namespace

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

int ok() {
  g_msg[0] = 0;
  return PF_OK;
}

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PF_OK;
  return fail(PF_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

int sm_count() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    n = 148;
  cache[dev] = n;
  return n;
}

int host_alias(void* host, void** dev) {
  cudaError_t e = cudaHostGetDevicePointer(dev, host, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PF_EINVAL, "host_out must be pinned host memory (%s)", cudaGetErrorString(e));
  }
  return PF_OK;
}

namespace {
std::atomic<int64_t> g_launches{0};

struct LaunchRec {
  const char* name;
  cudaEvent_t a, b;
};

struct Profiler {
  bool on = false;
  std::vector<LaunchRec> recs;
  std::vector<cudaEvent_t> pool;
  const char* pending_name = nullptr;
  cudaEvent_t pending = nullptr;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return e;
  }
};
thread_local Profiler g_prof;
}  // namespace

void launch_begin(const char* name, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!g_prof.on) return;
  g_prof.pending_name = name;
  g_prof.pending = g_prof.get();
  if (g_prof.pending) cudaEventRecord(g_prof.pending, st);
}

void launch_end(cudaStream_t st) {
  if (!g_prof.on || !g_prof.pending) return;
  cudaEvent_t b = g_prof.get();
  if (!b) return;
  cudaEventRecord(b, st);
  g_prof.recs.push_back(LaunchRec{g_prof.pending_name, g_prof.pending, b});
  g_prof.pending = nullptr;
}

int opt_in_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  if (bytes == 0) return PF_OK;
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{fn, dev}];
  if (have >= bytes) return PF_OK;
  // the limit covers dynamic + static shared memory
  cudaFuncAttributes fa{};
  PF_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (bytes + fa.sharedSizeBytes <= 48 * 1024) {
    have = bytes;
    return PF_OK;
  }
  PF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  have = bytes;
  return PF_OK;
}

int record_event(cudaStream_t st, cudaEvent_t* out) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  thread_local std::map<std::pair<int, cudaStream_t>, cudaEvent_t> events;
  cudaEvent_t ev;
  auto it = events.find({dev, st});
  if (it == events.end()) {
    PF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    events.emplace(std::make_pair(dev, st), ev);
  } else {
    ev = it->second;
  }
  PF_CUDA(cudaEventRecord(ev, st));
  *out = ev;
  return PF_OK;
}

int wait_event(cudaEvent_t ev) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t limit = g_wait_ms.load();
  int spins = 0;
  while (true) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return PF_OK;
    if (e != cudaErrorNotReady) return cuda_status(e, "waiting for the stream");
    if (++spins > 64) {
      const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                          std::chrono::steady_clock::now() - t0)
                          .count();
      if (ms > limit)
        return fail(PF_ETIMEOUT, "the stream did not reach the call's event within %lld ms",
                    (long long)limit);
      std::this_thread::sleep_for(std::chrono::microseconds(spins > 4096 ? 200 : 5));
    }
  }
}

int wait_stream(cudaStream_t st) {
  cudaEvent_t ev;
  int rc = record_event(st, &ev);
  if (rc != PF_OK) return rc;
  return wait_event(ev);
}

}  // namespace pf

extern "C" {

const char* pf_last_error(void) { return pf::g_msg; }

const char* pf_version(void) { return "0.1.0"; }

void pf_set_wait_timeout_ms(int64_t ms) { pf::g_wait_ms.store(ms > 0 ? ms : 1); }

int64_t pf_launch_count(void) { return pf::g_launches.load(); }

void pf_profile_begin(void) {
  pf::g_prof.on = true;
  for (auto& r : pf::g_prof.recs) {
    pf::g_prof.pool.push_back(r.a);
    pf::g_prof.pool.push_back(r.b);
  }
  pf::g_prof.recs.clear();
}

int pf_profile_end(int max_kernels, char* names, int name_len, double* total_ms,
                   int64_t* launches) {
  pf::g_prof.on = false;
  std::vector<std::pair<std::string, std::pair<double, int64_t>>> agg;
  for (auto& r : pf::g_prof.recs) {
    if (cudaEventSynchronize(r.b) != cudaSuccess) return pf::cuda_status(cudaGetLastError(), "profile");
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess)
      return pf::cuda_status(cudaGetLastError(), "profile");
    size_t i = 0;
    for (; i < agg.size(); ++i)
      if (agg[i].first == r.name) break;
    if (i == agg.size()) agg.push_back({r.name, {0.0, 0}});
    agg[i].second.first += ms;
    agg[i].second.second += 1;
  }
  const int n = (int)std::min<size_t>(agg.size(), (size_t)std::max(max_kernels, 0));
  for (int i = 0; i < n; ++i) {
    if (names && name_len > 0) {
      std::snprintf(names + (size_t)i * name_len, name_len, "%s", agg[i].first.c_str());
    }
    if (total_ms) total_ms[i] = agg[i].second.first;
    if (launches) launches[i] = agg[i].second.second;
  }
  for (auto& r : pf::g_prof.recs) {
    pf::g_prof.pool.push_back(r.a);
    pf::g_prof.pool.push_back(r.b);
  }
  pf::g_prof.recs.clear();
  pf::ok();
  return (int)agg.size();
}

int64_t pf_rows_per_unit(int64_t row_bytes) {
  if (row_bytes <= 0) return 1;
  int64_t a = row_bytes, b = 512;
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return 512 / a;
}

}  // extern "C"
