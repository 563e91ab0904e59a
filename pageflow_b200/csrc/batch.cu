// The batched join -> group-by: many independent instances of uneven size in
// one persistent launch fed by a device work queue.
//
// Layout (the workspace, laid out by pf_batch_prepare):
//   header       epoch, work counter, item totals, error word
//   descriptors  per instance: its columns, table region, slab, item ranges
//   remaining    per instance: build items not yet done
//   tables       per instance, 2 x build rows 16-byte slots {key, group | tag}
//   slabs        per instance, n_groups (sum, count) int64 pairs
//
// Work items, instance by instance: its build rows in items of BITEM rows,
// then its probe rows in items of PITEM rows (so the tables in use at any
// time are those of the few instances in flight, which stay in L2).  A block
// takes the next item from the counter; a probe item waits (bounded) until
// its instance's build items are all done.  Those items were taken before it,
// by blocks that are running, so the wait always ends.  A slot is free for this run when
// its tag is below the run's epoch; the claim is an atomicMax of the tag.
// Matches aggregate with warp-level combining of equal groups (hot keys of a
// skewed probe side become one atomic per warp, not one per row).
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "agg.cuh"

namespace pf {
namespace {

constexpr int BT2 = 256;
#ifndef PF_BATCH_BV
#define PF_BATCH_BV 1
#endif
// 1: the probe loop loads the next round's keys and values while this round
// probes its slots (loading two rounds ahead and prefetching the next
// round's first slots into L2 measured slower: 35.5 against 42.1 G rows/s)
#ifndef PF_BATCH_PIPE
#define PF_BATCH_PIPE 1
#endif
// rows a thread keeps in flight (all 4096 instances of the batch workload:
// 1 row 42.7 G rows/s, 2 rows 36.9, 4 rows 29.4: more registers a thread
// cost more resident warps than the extra loads in flight gain)
constexpr int BV = PF_BATCH_BV;
// 1: a probe item adds into the block's group cache (agg.cuh) and flushes it
// at the item's end, so the hot groups of a skewed instance cost one global
// atomic pair a block and item instead of one a warp and step; 0:
// warp-combined global atomics only.
#ifndef PF_BATCH_CACHE
#define PF_BATCH_CACHE 1
#endif
// with the cache: 1 combine equal groups of a warp before the cache
#ifndef PF_BATCH_CACHE_COMBINE
#define PF_BATCH_CACHE_COMBINE 0
#endif
constexpr size_t BATCH_SMEM = PF_BATCH_CACHE ? sizeof(GroupCache) : 0;
// Warp-combined add whose leaders go through the cache.
__device__ __forceinline__ void combined_to(GroupCache& gc, unsigned long long* slab, long long g,
                                            long long value) {
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, g);
  if (g < 0) return;
  const unsigned long long v = (unsigned long long)value;
  const unsigned s0 = __reduce_add_sync(peers, (unsigned)(v & 0x3fffff));
  const unsigned s1 = __reduce_add_sync(peers, (unsigned)((v >> 22) & 0x3fffff));
  const unsigned s2 = __reduce_add_sync(peers, (unsigned)(v >> 44));
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1)
    cache_add(gc, slab, g,
              (unsigned long long)s0 + ((unsigned long long)s1 << 22) +
                  ((unsigned long long)s2 << 44),
              (unsigned long long)__popc(peers));
}

constexpr int BITEM = 4096;
#ifndef PF_BATCH_PITEM
#define PF_BATCH_PITEM 16384
#endif
constexpr int PITEM = PF_BATCH_PITEM;
constexpr unsigned WAIT_LIMIT = 1u << 24;  // polls of a probe item's wait (x ~0.5 us)

struct Desc {
  const long long* bkey;
  const int* bgrp;
  long long nb;
  const long long* pfk;
  const long long* pval;
  long long np;
  long long gmin, ng;
  unsigned long long toff;   // first slot of the table region
  unsigned long long tcap;   // slots
  unsigned long long soff;   // first (sum, count) pair of the slab
  long long item0;             // first work item (its build items, then its probe items)
  long long nbi;               // build items
};

struct Header {
  unsigned epoch;
  unsigned pad;
  unsigned long long counter;
  long long n_build_items, n_items;
  int n_inst;
  int pad2;
  unsigned long long error;
};

struct Slot {
  unsigned long long key;
  unsigned long long tagged;  // (tag << 32) | group offset
};

struct Layout {
  Header* header;
  Desc* desc;
  unsigned* remaining;
  int* imap;  // work item -> instance
  Slot* tables;
  unsigned long long* slabs;
  unsigned long long table_slots, slab_pairs;
};

Layout layout(char* base, int n, unsigned long long table_slots, unsigned long long slab_pairs,
              unsigned long long items, size_t* used) {
  Arena a(base, ~(size_t)0);
  Layout l{};
  l.header = a.take<Header>(1);
  l.desc = a.take<Desc>(std::max(n, 1));
  l.remaining = a.take<unsigned>(std::max(n, 1));
  l.imap = a.take<int>(std::max<unsigned long long>(items, 1));
  l.tables = a.take<Slot>(std::max<unsigned long long>(table_slots, 1));
  l.slabs = a.take<unsigned long long>(2 * std::max<unsigned long long>(slab_pairs, 1));
  l.table_slots = table_slots;
  l.slab_pairs = slab_pairs;
  if (used) *used = a.used;
  return l;
}

void totals(const pf_batch_instance* in, int n, unsigned long long* ts, unsigned long long* sp,
            unsigned long long* items) {
  *ts = 0;
  *sp = 0;
  *items = 0;
  for (int i = 0; i < n; ++i) {
    const long long nb = std::max<int64_t>(in[i].n_build, 0);
    const long long np = nb > 0 ? std::max<int64_t>(in[i].n_probe, 0) : 0;
    *ts += 2ULL * (unsigned long long)nb;
    *sp += (unsigned long long)std::max<int64_t>(in[i].n_groups, 0);
    *items += (unsigned long long)((nb + BITEM - 1) / BITEM + (np + PITEM - 1) / PITEM);
  }
}

// Run start: bump the epoch, zero the counter, the error word and the slabs,
// and set every instance's remaining build items.
__global__ void k_batch_reset(Header* h, Desc* d, unsigned* remaining, int n,
                              unsigned long long* slabs, unsigned long long words) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (tid == 0) {
    h->epoch += 1;
    h->counter = 0;
    h->error = 0;
  }
  for (long long i = tid; i < n; i += stride) remaining[i] = (unsigned)d[i].nbi;
  for (long long i = tid; i < (long long)words; i += stride) slabs[i] = 0;
}

__device__ __forceinline__ unsigned first_slot(uint64_t h, unsigned long long cap) {
  return (unsigned)(((h >> 32) * cap) >> 32);
}

__global__ void __launch_bounds__(BT2) k_batch(Header* h, const Desc* d, const int* __restrict__ imap,
                                               unsigned* remaining,
                                               Slot* tables, unsigned long long* slabs,
                                               unsigned long long* stats) {
  __shared__ long long item_s;
  __shared__ int ok_s;
  const unsigned epoch = h->epoch;
  const long long ni = h->n_items;
  unsigned long long matched = 0, bad_group = 0, overflow = 0;
#if PF_BATCH_CACHE
  extern __shared__ __align__(16) unsigned char batch_smem[];
  GroupCache& gc = *reinterpret_cast<GroupCache*>(batch_smem);
  cache_init(gc);
#endif
  // With PF_PREFETCH_ITEMS, thread 0 takes the block's next item while the
  // block works on the current one (measured no faster, so off by default).
  // Items are taken in increasing order and an item waits only for items
  // before it, so the smallest unfinished item is always some block's
  // current item with nothing left to wait for: the launch progresses.
  if (threadIdx.x == 0) item_s = (long long)atomicAdd(&h->counter, 1ULL);
  while (true) {
    __syncthreads();
    const long long it = item_s;
    if (it >= ni) break;
    unsigned long long next = 0;
    if (PF_PREFETCH_ITEMS && threadIdx.x == 0) next = atomicAdd(&h->counter, 1ULL);
    const int inst = imap[it];
    // the instance's descriptor in registers for the item (read through a
    // reference, every store to the tables or slabs would reload it)
    const Desc D = d[inst];
    const long long local = it - D.item0;
    if (local < D.nbi) {
      // BV rows a thread at a time: loads, then every first claim, then the
      // (rare) collisions
      const long long lo = local * BITEM, hi = min(D.nb, lo + BITEM);
      for (long long i0 = lo; i0 < hi; i0 += BT2 * BV) {
        unsigned long long key[BV];
        uint32_t goff[BV];
        unsigned pos[BV];
        bool live[BV], done[BV];
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          const long long i = i0 + k * BT2 + threadIdx.x;
          live[k] = i < hi;
          key[k] = live[k] ? (unsigned long long)D.bkey[i] : 0ULL;
          const long long g = live[k] ? (long long)D.bgrp[i] - D.gmin : 0;
          goff[k] = 0xffffffffu;
          if (g >= 0 && g < D.ng) goff[k] = (uint32_t)g;
          else if (live[k]) ++bad_group;
        }
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          pos[k] = first_slot(mix64(key[k]), D.tcap);
          done[k] = false;
          if (!live[k]) continue;
          Slot* sl = tables + D.toff + pos[k];
          unsigned* tag = reinterpret_cast<unsigned*>(&sl->tagged) + 1;
          if (atomicMax(tag, epoch) < epoch) {
            *reinterpret_cast<ulonglong2*>(sl) =
                make_ulonglong2(key[k], ((unsigned long long)epoch << 32) | goff[k]);
            done[k] = true;
          }
        }
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          if (!live[k] || done[k]) continue;
          unsigned p = pos[k];
          for (unsigned long long left = D.tcap - 1; left > 0; --left) {
            if (++p == D.tcap) p = 0;
            Slot* sl = tables + D.toff + p;
            unsigned* tag = reinterpret_cast<unsigned*>(&sl->tagged) + 1;
            if (atomicMax(tag, epoch) < epoch) {
              *reinterpret_cast<ulonglong2*>(sl) =
                  make_ulonglong2(key[k], ((unsigned long long)epoch << 32) | goff[k]);
              done[k] = true;
              break;
            }
          }
          overflow += !done[k];
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicSub(&remaining[inst], 1u);
      }
    } else {
      if (threadIdx.x == 0) {
        unsigned polls = 0;
        while (ld_acquire_u32(&remaining[inst]) != 0 && polls < WAIT_LIMIT) {
          __nanosleep(256);
          ++polls;
        }
        ok_s = polls < WAIT_LIMIT;
        if (!ok_s) atomicOr(&h->error, 1ULL);
        __threadfence();
      }
      __syncthreads();
      if (!ok_s) {
        if (threadIdx.x == 0) item_s = (long long)(PF_PREFETCH_ITEMS ? next : atomicAdd(&h->counter, 1ULL));
        continue;
      }
      // BV rows a thread at a time: keys, then every first slot and value,
      // then the (rare) collisions
      const long long lo = (local - D.nbi) * PITEM, hi = min(D.np, lo + PITEM);
#if PF_BATCH_PIPE
      // the next round's keys and values load while this round probes
      unsigned long long key[BV];
      long long value[BV];
#pragma unroll
      for (int k = 0; k < BV; ++k) {
        const long long i = lo + k * BT2 + threadIdx.x;
        const bool l = i < hi && D.tcap > 0;
        key[k] = l ? (unsigned long long)D.pfk[i] : 0ULL;
        value[k] = l ? D.pval[i] : 0;
      }
#endif
      for (long long i0 = lo; i0 < hi; i0 += BT2 * BV) {
        unsigned pos[BV];
        ulonglong2 sl[BV];
        long long g[BV];
        bool live[BV];
#if PF_BATCH_PIPE
        unsigned long long nkey[BV];
        long long nval[BV];
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          const long long i = i0 + (long long)BT2 * BV + k * BT2 + threadIdx.x;
          const bool l = i < hi && D.tcap > 0;
          nkey[k] = l ? (unsigned long long)D.pfk[i] : 0ULL;
          nval[k] = l ? D.pval[i] : 0;
        }
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          live[k] = i0 + k * BT2 + threadIdx.x < hi && D.tcap > 0;
          pos[k] = live[k] ? first_slot(mix64(key[k]), D.tcap) : 0u;
          sl[k] = live[k] ? __ldcg(reinterpret_cast<const ulonglong2*>(tables + D.toff + pos[k]))
                          : make_ulonglong2(0ULL, 0ULL);
        }
#else
        unsigned long long key[BV];
        long long value[BV];
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          const long long i = i0 + k * BT2 + threadIdx.x;
          live[k] = i < hi && D.tcap > 0;
          key[k] = live[k] ? (unsigned long long)D.pfk[i] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          const long long i = i0 + k * BT2 + threadIdx.x;
          pos[k] = live[k] ? first_slot(mix64(key[k]), D.tcap) : 0u;
          sl[k] = live[k] ? __ldcg(reinterpret_cast<const ulonglong2*>(tables + D.toff + pos[k]))
                          : make_ulonglong2(0ULL, 0ULL);
          value[k] = live[k] ? D.pval[i] : 0;
        }
#endif
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          g[k] = -1;
          if (!live[k]) continue;
          ulonglong2 x = sl[k];
          unsigned p = pos[k];
          for (unsigned long long probes = 0; probes < D.tcap; ++probes) {
            if ((uint32_t)(x.y >> 32) != epoch) break;
            if (x.x == key[k]) {
              ++matched;
              const uint32_t go = (uint32_t)x.y;
              if (go != 0xffffffffu) g[k] = go;
              break;
            }
            if (++p == D.tcap) p = 0;
            x = __ldcg(reinterpret_cast<const ulonglong2*>(tables + D.toff + p));
          }
        }
#pragma unroll
        for (int k = 0; k < BV; ++k) {
#if PF_BATCH_CACHE && PF_BATCH_CACHE_COMBINE
          combined_to(gc, slabs + 2 * D.soff, g[k], g[k] >= 0 ? value[k] : 0);
#elif PF_BATCH_CACHE
          if (g[k] >= 0) cache_add(gc, slabs + 2 * D.soff, g[k], (unsigned long long)value[k], 1ULL);
#else
          combined_add(slabs + 2 * D.soff, g[k], g[k] >= 0 ? value[k] : 0);
#endif
        }
#if PF_BATCH_PIPE
#pragma unroll
        for (int k = 0; k < BV; ++k) {
          key[k] = nkey[k];
          value[k] = nval[k];
        }
#endif
      }
#if PF_BATCH_CACHE
      cache_flush(gc, slabs + 2 * D.soff);
#endif
    }
    __syncthreads();  // every thread has read item_s
    if (threadIdx.x == 0) item_s = (long long)(PF_PREFETCH_ITEMS ? next : atomicAdd(&h->counter, 1ULL));
  }
  for (int o = 16; o; o >>= 1) matched += __shfl_xor_sync(FULL, matched, o);
  if ((threadIdx.x & 31) == 0 && matched) atomicAdd(&stats[0], matched);
  if (bad_group) atomicAdd(&stats[2], bad_group);
  if (overflow) atomicAdd(&stats[3], overflow);
}

__global__ void k_batch_error(const Header* h, unsigned long long* stats) {
  if (threadIdx.x == 0 && h->error) stats[1] |= h->error;
}

// What pf_batch_run and pf_batch_slab need of a prepared workspace, kept on
// the host (keyed by the workspace's address) so that a run touches no host
// copy of device memory and can be captured.
struct HostPlan {
  int n = 0;
  unsigned long long table_slots = 0, slab_pairs = 0, items = 0;
  std::vector<unsigned long long> slab_off;
};

std::mutex g_plans_mu;
std::map<void*, HostPlan> g_plans;

bool find_plan(void* ws, HostPlan* out) {
  std::lock_guard<std::mutex> lock(g_plans_mu);
  auto it = g_plans.find(ws);
  if (it == g_plans.end()) return false;
  *out = it->second;
  return true;
}

// The persistent grid: every block resident at once.
int batch_grid(int* grid) {
  int per_sm = 0;
  if (int rc = opt_in_smem((const void*)k_batch, BATCH_SMEM)) return rc;
  PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, BT2, BATCH_SMEM));
  *grid = std::max(1, per_sm) * sm_count();
  return PF_OK;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_batch_workspace(const pf_batch_instance* in, int n) {
  unsigned long long ts, sp, items;
  totals(in, n, &ts, &sp, &items);
  size_t used = 0;
  layout(nullptr, n, ts, sp, items, &used);
  return used + 256;
}

extern "C" int pf_batch_prepare(const pf_batch_instance* in, int n, void* workspace,
                                size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 1) return fail(PF_EINVAL, "batch: at least one instance");
  unsigned long long ts, sp, items;
  totals(in, n, &ts, &sp, &items);
  size_t used = 0;
  Layout l = layout((char*)workspace, n, ts, sp, items, &used);
  if (!workspace || used > workspace_bytes || ((uintptr_t)workspace & 255))
    return fail(PF_ENOSPACE,
                "batch: workspace of %zu bytes at %p, %zu needed on a 256-byte boundary",
                workspace_bytes, workspace, used);
  std::vector<Desc> d(n);
  unsigned long long toff = 0, soff = 0;
  long long bi = 0, pi = 0;
  for (int i = 0; i < n; ++i) {
    const pf_batch_instance& x = in[i];
    if (x.n_build < 0 || x.n_probe < 0 || x.n_groups < 0 || x.n_groups > 0xfffffffeLL)
      return fail(PF_EINVAL, "batch: instance %d has bad sizes", i);
    if ((x.n_build > 0 && (!x.build_key || !x.build_group)) ||
        (x.n_probe > 0 && (!x.probe_fk || !x.probe_value)))
      return fail(PF_EINVAL, "batch: instance %d has a null column", i);
    Desc& D = d[i];
    D.bkey = (const long long*)x.build_key;
    D.bgrp = x.build_group;
    D.nb = x.n_build;
    D.pfk = (const long long*)x.probe_fk;
    D.pval = (const long long*)x.probe_value;
    // no build rows or no groups: nothing can match or be aggregated
    D.np = (x.n_build > 0) ? x.n_probe : 0;
    D.gmin = x.group_min;
    D.ng = x.n_groups;
    D.toff = toff;
    D.tcap = 2ULL * (unsigned long long)x.n_build;
    if (D.tcap > 0xffffffffULL) return fail(PF_EINVAL, "batch: instance %d is over 2^31 build rows", i);
    D.soff = soff;
    D.item0 = bi + pi;
    D.nbi = (D.nb + BITEM - 1) / BITEM;
    toff += D.tcap;
    soff += (unsigned long long)x.n_groups;
    bi += (D.nb + BITEM - 1) / BITEM;
    pi += (D.np + PITEM - 1) / PITEM;
  }
  Header hh{};
  hh.epoch = 0;
  hh.counter = 0;
  hh.n_build_items = bi;
  hh.n_items = bi + pi;
  hh.n_inst = n;
  if ((unsigned long long)(bi + pi) != items)
    return fail(PF_EINVAL, "batch: %lld work items, %llu planned", bi + pi, items);
  std::vector<int> imap((size_t)std::max<unsigned long long>(items, 1), 0);
  for (int i = 0; i < n; ++i) {
    const long long nit = d[i].nbi + (d[i].np + PITEM - 1) / PITEM;
    for (long long k = 0; k < nit; ++k) imap[(size_t)(d[i].item0 + k)] = i;
  }
  PF_CUDA(cudaMemcpyAsync(l.imap, imap.data(), sizeof(int) * imap.size(), cudaMemcpyHostToDevice,
                          st));
  PF_CUDA(cudaMemcpyAsync(l.desc, d.data(), sizeof(Desc) * n, cudaMemcpyHostToDevice, st));
  PF_CUDA(cudaMemcpyAsync(l.header, &hh, sizeof(Header), cudaMemcpyHostToDevice, st));
  PF_CUDA(cudaMemsetAsync(l.tables, 0, sizeof(Slot) * std::max<unsigned long long>(ts, 1), st));
  if (int rc = wait_stream(st)) return rc;  // the host copies above read d and hh
  HostPlan hp;
  hp.n = n;
  hp.table_slots = ts;
  hp.slab_pairs = sp;
  hp.items = items;
  hp.slab_off.resize(n);
  for (int i = 0; i < n; ++i) hp.slab_off[i] = d[i].soff;
  {
    std::lock_guard<std::mutex> lock(g_plans_mu);
    g_plans[workspace] = std::move(hp);
  }
  return ok();
}

extern "C" int pf_batch_run(void* workspace, int64_t* stats, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  HostPlan hp;
  if (!find_plan(workspace, &hp)) return fail(PF_EINVAL, "batch: workspace was not prepared");
  if (!stats) return fail(PF_EINVAL, "batch: null stats");
  Layout l = layout((char*)workspace, hp.n, hp.table_slots, hp.slab_pairs, hp.items, nullptr);
  int grid = 0;
  if (int rc = batch_grid(&grid)) return rc;
  PF_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(int64_t), st));
  {
    PF_KERNEL("k_batch_reset", st);
    const long long words = 2LL * (long long)hp.slab_pairs;
    const unsigned g = (unsigned)std::max<long long>(
        1, std::min<long long>((words + 255) / 256, (long long)sm_count() * 8));
    k_batch_reset<<<g, 256, 0, st>>>(l.header, l.desc, l.remaining, hp.n, l.slabs,
                                      (unsigned long long)words);
  }
  PF_LAUNCH("k_batch_reset");
  {
    PF_KERNEL("k_batch", st);
    k_batch<<<grid, BT2, BATCH_SMEM, st>>>(l.header, l.desc, l.imap, l.remaining, l.tables, l.slabs,
                                  (unsigned long long*)stats);
  }
  PF_LAUNCH("k_batch");
  {
    PF_KERNEL("k_batch_error", st);
    k_batch_error<<<1, 32, 0, st>>>(l.header, (unsigned long long*)stats);
  }
  PF_LAUNCH("k_batch_error");
  return ok();
}

extern "C" int64_t* pf_batch_slab(void* workspace, int i) {
  HostPlan hp;
  if (!find_plan(workspace, &hp) || i < 0 || i >= hp.n) return nullptr;
  Layout l = layout((char*)workspace, hp.n, hp.table_slots, hp.slab_pairs, hp.items, nullptr);
  return (int64_t*)(l.slabs + 2 * hp.slab_off[i]);
}
