// Seeded synthetic join workloads generated on the device (synth.h holds the
// generator; the CPU twin in the oracle includes the same header).
#include "common.cuh"
#include "synth.h"

namespace pf {
namespace {

__global__ void k_gen_build(uint64_t seed, uint64_t n_build, uint64_t n_groups, pf_perm_t perm,
                            long long lo, long long rows, long long* __restrict__ key,
                            int* __restrict__ group) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (long long)gridDim.x * blockDim.x) {
    int64_t k;
    int32_t g;
    pf_gen_build_row(seed, n_build, n_groups, &perm, (uint64_t)(lo + i), &k, &g);
    key[i] = k;
    group[i] = g;
  }
}

__global__ void k_gen_probe(uint64_t seed, uint64_t n_build, int miss, long long lo,
                            long long rows, long long* __restrict__ fk,
                            long long* __restrict__ price, long long* __restrict__ disc) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (long long)gridDim.x * blockDim.x) {
    int64_t f, p, d;
    pf_gen_probe_row(seed, n_build, miss, (uint64_t)(lo + i), &f, &p, &d);
    fk[i] = f;
    price[i] = p;
    disc[i] = d;
  }
}

__global__ void k_gen_batch_probe(uint64_t seed, pf_perm_t perm, int nbins,
                                  const int64_t* __restrict__ edges,
                                  const uint64_t* __restrict__ thr, long long lo, long long rows,
                                  long long* __restrict__ fk, long long* __restrict__ value) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (long long)gridDim.x * blockDim.x) {
    int64_t f, v;
    pf_gen_batch_probe_row(seed, &perm, nbins, edges, thr, (uint64_t)(lo + i), &f, &v);
    fk[i] = f;
    value[i] = v;
  }
}

__global__ void k_gen_serve_dim(uint64_t gseed, pf_perm_t perm, uint64_t n_groups, long long lo,
                                long long rows, long long* __restrict__ key,
                                int* __restrict__ group) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (long long)gridDim.x * blockDim.x) {
    int64_t k;
    int32_t g;
    pf_gen_serve_dim_row(gseed, &perm, n_groups, (uint64_t)(lo + i), &k, &g);
    key[i] = k;
    group[i] = g;
  }
}

__global__ void k_gen_serve_fact(uint64_t seed, pf_perm_t perm, int nbins,
                                 const int64_t* __restrict__ edges,
                                 const uint64_t* __restrict__ thr, long long lo, long long rows,
                                 long long* __restrict__ fk, int* __restrict__ date,
                                 long long* __restrict__ value) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (long long)gridDim.x * blockDim.x) {
    int64_t f, v;
    int32_t d;
    pf_gen_serve_fact_row(seed, &perm, nbins, edges, thr, (uint64_t)(lo + i), &f, &d, &v);
    fk[i] = f;
    date[i] = d;
    value[i] = v;
  }
}

unsigned grid_for(long long rows) {
  const long long want = (rows + 255) / 256;
  const long long cap = (long long)sm_count() * 16;
  return (unsigned)std::max<long long>(1, std::min(want, cap));
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int pf_gen_build(int config, uint64_t seed, int64_t n_build, int64_t n_groups,
                            int64_t lo, int64_t rows, int64_t* key, int32_t* group, void* stream) {
  if (n_build < 1 || n_groups < 1 || lo < 0 || rows < 0 || lo + rows > n_build)
    return fail(PF_EINVAL, "gen_build: rows [%lld, %lld) outside a build of %lld",
                (long long)lo, (long long)(lo + rows), (long long)n_build);
  (void)config;
  if (rows == 0) return ok();
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  {
    PF_KERNEL("k_gen_build", (cudaStream_t)stream);
    k_gen_build<<<grid_for(rows), 256, 0, (cudaStream_t)stream>>>(
        seed, (uint64_t)n_build, (uint64_t)n_groups, perm, lo, rows, (long long*)key, group);
  }
  PF_LAUNCH("k_gen_build");
  return ok();
}

extern "C" int pf_gen_batch_probe(uint64_t seed, int64_t n_build, int64_t lo, int64_t rows,
                                  int nbins, const int64_t* edges, const uint64_t* thr,
                                  int64_t* fk, int64_t* value, void* stream) {
  if (n_build < 1 || lo < 0 || rows < 0 || nbins < 1)
    return fail(PF_EINVAL, "gen_batch_probe: bad arguments");
  if (rows == 0) return ok();
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  {
    PF_KERNEL("k_gen_batch_probe", (cudaStream_t)stream);
    k_gen_batch_probe<<<grid_for(rows), 256, 0, (cudaStream_t)stream>>>(
        seed, perm, nbins, edges, thr, lo, rows, (long long*)fk, (long long*)value);
  }
  PF_LAUNCH("k_gen_batch_probe");
  return ok();
}

extern "C" int pf_gen_probe(int config, uint64_t seed, int64_t n_build, int64_t lo, int64_t rows,
                            int64_t* fk, int64_t* price, int64_t* disc, void* stream) {
  if (n_build < 1 || lo < 0 || rows < 0)
    return fail(PF_EINVAL, "gen_probe: bad arguments");
  if (rows == 0) return ok();
  {
    PF_KERNEL("k_gen_probe", (cudaStream_t)stream);
    k_gen_probe<<<grid_for(rows), 256, 0, (cudaStream_t)stream>>>(
        seed, (uint64_t)n_build, pf_cfg_miss_per_10(config), lo, rows, (long long*)fk,
        (long long*)price, (long long*)disc);
  }
  PF_LAUNCH("k_gen_probe");
  return ok();
}

extern "C" int pf_gen_serve_dim(uint64_t seed, int64_t n_ranks, uint64_t group_seed,
                                int64_t n_keys, int64_t n_groups, int64_t lo, int64_t rows,
                                int64_t* key, int32_t* group, void* stream) {
  if (n_ranks < 1 || n_keys < 1 || n_keys > n_ranks || n_groups < 1 || n_groups > INT32_MAX ||
      lo < 0 || rows < 0 || lo + rows > n_keys)
    return fail(PF_EINVAL, "gen_serve_dim: bad arguments");
  if (rows == 0) return ok();
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_ranks);
  {
    PF_KERNEL("k_gen_serve_dim", (cudaStream_t)stream);
    k_gen_serve_dim<<<grid_for(rows), 256, 0, (cudaStream_t)stream>>>(
        group_seed, perm, (uint64_t)n_groups, lo, rows, (long long*)key, group);
  }
  PF_LAUNCH("k_gen_serve_dim");
  return ok();
}

extern "C" int pf_gen_serve_fact(uint64_t seed, int64_t n_ranks, int nbins, const int64_t* edges,
                                 const uint64_t* thr, int64_t lo, int64_t rows, int64_t* fk,
                                 int32_t* date, int64_t* value, void* stream) {
  if (n_ranks < 1 || lo < 0 || rows < 0 || nbins < 1)
    return fail(PF_EINVAL, "gen_serve_fact: bad arguments");
  if (rows == 0) return ok();
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_ranks);
  {
    PF_KERNEL("k_gen_serve_fact", (cudaStream_t)stream);
    k_gen_serve_fact<<<grid_for(rows), 256, 0, (cudaStream_t)stream>>>(
        seed, perm, nbins, edges, thr, lo, rows, (long long*)fk, date, (long long*)value);
  }
  PF_LAUNCH("k_gen_serve_fact");
  return ok();
}
