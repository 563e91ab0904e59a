// The join cores, sm_100a replacements of tqpkernels.join_unique_hash,
// join_semi_anti and join_expand (reference operators/kernels/join_core.cu,
// wrapper operators/join_core.py):
//
//   unique hash  inner join on a build tuple (1-2 int64 keys) proven unique:
//                a table of 2*n_build 4-byte slots (the build row in the low
//                r bits, r the bit width of n_build; the tuple hash's bits
//                above them as a fingerprint), linear probing; each probe
//                row's partner; the matched probe rows compacted in order
//   semi / anti  a set of the build keys (INT64_MIN marks an empty slot), with
//                an optional per-key min / max of one build column answering
//                a residual comparison; the kept probe rows compacted in order
//   expand       the pairs of the sort/search probe: each probe row's run of
//                equal build keys, in probe-row order
//
// Slots come from the tuple hash's bits just below its top nine (the radix
// bucket's bits, B <= 512, are shared by a bucket's keys).  Every kernel
// bounds its probe loop by the table's size.  Each call queues its kernels,
// writes its row count into the caller's pinned host_out through the device
// alias, and waits for that count once.
#include <climits>
#include <mutex>

#include "scan.cuh"

namespace pf {
namespace {

constexpr int T = 256;
constexpr unsigned EMPTY_SLOT = ~0u;
constexpr long long EMPTY_KEY = LLONG_MIN;

__device__ __forceinline__ uint64_t tuple_hash(long long k0, long long k1, bool two) {
  uint64_t h = mix64((uint64_t)k0);
  if (two) h = mix64(h ^ (mix64((uint64_t)k1) + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2)));
  return h;
}

// The first slot of a hash among 2^logcap: the bits right below its top nine.
__device__ __forceinline__ uint64_t first_slot(uint64_t h, int logcap) {
  return (h << 9) >> (64 - logcap);
}

// ---- unique hash -------------------------------------------------------------
//
// A slot holds (hash << r) | row, rmask = 2^r - 1 with n_build <= rmask: a
// row never fills its r bits, so no entry is all ones (EMPTY_SLOT).  The home
// slot is the multiply-shift of the hash's bits below its top nine onto
// [0, cap) (reference operators/kernels/join_core.cu:55 slot_of), which
// leans on the high bits; the fingerprint takes the low ones.

struct UhTable {
  unsigned* slot;
  unsigned long long cap;
  unsigned rmask;
  int rbits;
};

__device__ __forceinline__ unsigned long long uh_home(uint64_t h, unsigned long long cap) {
  return __umul64hi(h << 9, cap);
}

__device__ __forceinline__ unsigned long long uh_next(unsigned long long s,
                                                      unsigned long long cap) {
  return s + 1 == cap ? 0 : s + 1;
}

template <bool TWO>
__global__ void __launch_bounds__(T) k_uh_build(const long long* __restrict__ b0,
                                                const long long* __restrict__ b1, long long n,
                                                UhTable t) {
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n) return;
  const uint64_t h = tuple_hash(b0[i], TWO ? b1[i] : 0, TWO);
  const unsigned entry = ((unsigned)h << t.rbits) | (unsigned)i;
  unsigned long long s = uh_home(h, t.cap);
  for (unsigned long long probes = 0; probes < t.cap; ++probes) {
    if (atomicCAS(&t.slot[s], EMPTY_SLOT, entry) == EMPTY_SLOT) return;
    s = uh_next(s, t.cap);
  }
}

#ifndef PF_UH_U
#define PF_UH_U 2
#endif
constexpr int UH_U = PF_UH_U;  // probe rows a thread resolves together
static_assert(CITEMS % UH_U == 0, "probe batches tile a thread's rows");

// Probe CB rows a block: partner[i] (build row or -1), the block's matches.
// UH_U rows at a time: their home and next slots loaded together, then their
// candidates' keys; a row that those two slots do not settle walks on.
template <bool TWO>
__global__ void __launch_bounds__(CT) k_uh_probe(const long long* __restrict__ b0,
                                                 const long long* __restrict__ b1,
                                                 const long long* __restrict__ p0,
                                                 const long long* __restrict__ p1, long long n,
                                                 UhTable t, int* __restrict__ partner,
                                                 long long* __restrict__ bcnt) {
  const unsigned* __restrict__ tab = t.slot;
  const unsigned fmask = ~t.rmask;
  const long long base = (long long)blockIdx.x * CB;
  int c = 0;
  for (int kk = 0; kk < CITEMS; kk += UH_U) {
    long long k0[UH_U], k1[UH_U];
    unsigned fp[UH_U], e0[UH_U], e1[UH_U];
    unsigned long long s0[UH_U];
    int cand[UH_U], r[UH_U];
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      const long long i = base + (kk + u) * CT + threadIdx.x;
      k0[u] = i < n ? p0[i] : 0;
      k1[u] = TWO && i < n ? p1[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      const uint64_t h = tuple_hash(k0[u], k1[u], TWO);
      fp[u] = (unsigned)h << t.rbits;
      s0[u] = uh_home(h, t.cap);
    }
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      const bool in = base + (kk + u) * CT + threadIdx.x < n;
      e0[u] = in ? tab[s0[u]] : EMPTY_SLOT;
      e1[u] = in ? tab[uh_next(s0[u], t.cap)] : EMPTY_SLOT;
    }
    // the candidate among the two slots: -1 settled as no match, -2 walk on
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      if (e0[u] == EMPTY_SLOT) cand[u] = -1;
      else if ((e0[u] & fmask) == fp[u]) cand[u] = (int)(e0[u] & t.rmask);
      else if (e1[u] == EMPTY_SLOT) cand[u] = -1;
      else if ((e1[u] & fmask) == fp[u]) cand[u] = (int)(e1[u] & t.rmask);
      else cand[u] = -2;
    }
    long long c0[UH_U], c1[UH_U];
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      c0[u] = cand[u] >= 0 ? b0[cand[u]] : 0;
      c1[u] = TWO && cand[u] >= 0 ? b1[cand[u]] : 0;
    }
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      r[u] = -1;
      if (cand[u] >= 0 && c0[u] == k0[u] && (!TWO || c1[u] == k1[u])) r[u] = cand[u];
      else if (cand[u] != -1) {
        // a fingerprint that matched another key, or two full slots: walk
        // the chain from its home slot
        unsigned long long s = s0[u];
        for (unsigned long long probes = 0; probes < t.cap; ++probes) {
          const unsigned e = tab[s];
          if (e == EMPTY_SLOT) break;
          if ((e & fmask) == fp[u]) {
            const int row = (int)(e & t.rmask);
            if (b0[row] == k0[u] && (!TWO || b1[row] == k1[u])) {
              r[u] = row;
              break;
            }
          }
          s = uh_next(s, t.cap);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UH_U; ++u) {
      const long long i = base + (kk + u) * CT + threadIdx.x;
      if (i < n) {
        partner[i] = r[u];
        c += r[u] >= 0;
      }
    }
  }
  __shared__ int red[CT / 32];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int q = 0; q < CT / 32; ++q) s += red[q];
    bcnt[blockIdx.x] = s;
  }
}

// The matched probe rows of each block, in order, from the block's offset.
__global__ void __launch_bounds__(CT) k_uh_emit(const int* __restrict__ partner, long long n,
                                                const long long* __restrict__ boff,
                                                long long* __restrict__ build_idx,
                                                long long* __restrict__ probe_idx) {
  __shared__ int wsum[CT / 32];
  const long long base = (long long)blockIdx.x * CB + (long long)threadIdx.x * CITEMS;
  bool keep[CITEMS];
  int part[CITEMS], rank[CITEMS];
  if (base + CITEMS <= n) {
    const int4* v = reinterpret_cast<const int4*>(partner + base);
#pragma unroll
    for (int q = 0; q < CITEMS / 4; ++q) {
      const int4 x = v[q];
      part[4 * q] = x.x;
      part[4 * q + 1] = x.y;
      part[4 * q + 2] = x.z;
      part[4 * q + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < CITEMS; ++k) part[k] = base + k < n ? partner[base + k] : -1;
  }
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) keep[k] = part[k] >= 0;
  __shared__ unsigned short rows[CB];
  __shared__ int sp[CB];
  const int tot = block_ranks(keep, rank, wsum);
#pragma unroll
  for (int k = 0; k < CITEMS; ++k) {
    if (keep[k]) {
      rows[rank[k]] = (unsigned short)(threadIdx.x * CITEMS + k);
      sp[rank[k]] = part[k];
    }
  }
  __syncthreads();
  const long long o = boff[blockIdx.x], b0 = (long long)blockIdx.x * CB;
  for (int e = threadIdx.x; e < tot; e += CT) {
    build_idx[o + e] = sp[e];
    probe_idx[o + e] = b0 + rows[e];
  }
}

// ---- semi / anti ----------------------------------------------------------------

__global__ void __launch_bounds__(T) k_set_build(const long long* __restrict__ key,
                                                 const long long* __restrict__ val, long long n,
                                                 long long* table, long long* mn, long long* mx,
                                                 int logcap, long long* bad) {
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n) return;
  const long long k = key[i];
  if (k == EMPTY_KEY) {
    *bad = 1;
    return;
  }
  const uint64_t mask = (1ULL << logcap) - 1;
  uint64_t s = first_slot(mix64((uint64_t)k), logcap);
  bool in = false;
  for (uint64_t probes = 0; probes <= mask; ++probes) {
    long long cur = table[s];
    if (cur == EMPTY_KEY)
      cur = (long long)atomicCAS((unsigned long long*)&table[s], (unsigned long long)EMPTY_KEY,
                                 (unsigned long long)k);
    if (cur == EMPTY_KEY || cur == k) {
      in = true;
      break;
    }
    s = (s + 1) & mask;
  }
  if (!in) {
    *bad = 2;  // the set is full: cannot happen at half load
    return;
  }
  if (mn || mx) {
    const long long v = val[i];
    if (mn && v < mn[s]) atomicMin(&mn[s], v);
    if (mx && v > mx[s]) atomicMax(&mx[s], v);
  }
}

__global__ void __launch_bounds__(CT) k_set_probe(const long long* __restrict__ key,
                                                  const long long* __restrict__ val, long long n,
                                                  const long long* __restrict__ table,
                                                  const long long* __restrict__ mn,
                                                  const long long* __restrict__ mx, int logcap,
                                                  int op, bool anti, unsigned char* __restrict__ keep,
                                                  long long* __restrict__ bcnt) {
  const uint64_t mask = (1ULL << logcap) - 1;
  const long long base = (long long)blockIdx.x * CB;
  int c = 0;
  for (int k = 0; k < CITEMS; ++k) {
    const long long i = base + k * CT + threadIdx.x;
    if (i >= n) break;
    const long long kk = key[i];
    bool hit = false;
    uint64_t s = first_slot(mix64((uint64_t)kk), logcap);
    if (kk != EMPTY_KEY) {
      for (uint64_t probes = 0; probes <= mask; ++probes) {
        const long long t = table[s];
        if (t == kk) {
          hit = true;
          break;
        }
        if (t == EMPTY_KEY) break;
        s = (s + 1) & mask;
      }
    }
    if (hit && op != PF_OP_NONE) {
      const long long v = val[i];
      switch (op) {
        case PF_OP_NE: hit = mn[s] != v || mx[s] != v; break;
        case PF_OP_LT: hit = mn[s] < v; break;
        case PF_OP_LE: hit = mn[s] <= v; break;
        case PF_OP_GT: hit = mx[s] > v; break;
        default: hit = mx[s] >= v; break;
      }
    }
    const bool kp = hit != anti;
    keep[i] = kp;
    c += kp;
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

__global__ void __launch_bounds__(CT) k_keep_emit(const unsigned char* __restrict__ keep,
                                                  long long n, const long long* __restrict__ boff,
                                                  long long* __restrict__ out) {
  __shared__ int wsum[CT / 32];
  const long long base = (long long)blockIdx.x * CB + (long long)threadIdx.x * CITEMS;
  bool kp[CITEMS];
  int rank[CITEMS];
  if (base + CITEMS <= n) {
    const uint4 x = *reinterpret_cast<const uint4*>(keep + base);
    const unsigned w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int k = 0; k < CITEMS; ++k) kp[k] = ((w[k / 4] >> (8 * (k % 4))) & 0xffu) != 0;
  } else {
#pragma unroll
    for (int k = 0; k < CITEMS; ++k) kp[k] = base + k < n && keep[base + k];
  }
  __shared__ unsigned short rows[CB];
  const int tot = block_compact(kp, rank, rows, wsum);
  const long long o = boff[blockIdx.x], b0 = (long long)blockIdx.x * CB;
  for (int e = threadIdx.x; e < tot; e += CT) out[o + e] = b0 + rows[e];
}

__global__ void k_fill_i64(long long* p, long long v, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// ---- expand ---------------------------------------------------------------------

constexpr int EITEMS = 8;

// Thread t covers pairs [t*EITEMS, t*EITEMS + EITEMS): one binary search for
// the probe row of its first pair, then a walk.
__global__ void __launch_bounds__(T) k_expand(const long long* __restrict__ sorted_ids,
                                              const long long* __restrict__ start,
                                              const long long* __restrict__ len,
                                              const long long* __restrict__ incl, long long m,
                                              long long n_pairs, long long* __restrict__ cs,
                                              long long* __restrict__ cr) {
  const long long k0 = ((long long)blockIdx.x * T + threadIdx.x) * EITEMS;
  if (k0 >= n_pairs) return;
  long long lo = 0, hi = m - 1;  // first i with incl[i] > k0
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (incl[mid] <= k0) lo = mid + 1;
    else hi = mid;
  }
  long long i = lo;
  long long end = incl[i];
  for (int e = 0; e < EITEMS; ++e) {
    const long long k = k0 + e;
    if (k >= n_pairs) break;
    while (end <= k && i + 1 < m) end = incl[++i];
    const long long first = end - len[i];
    cs[k] = sorted_ids[start[i] + (k - first)];
    cr[k] = i;
  }
}

struct UhLayout {
  UhTable table;
  int* partner;
  long long* bcnt;
  long long* total;
};

UhLayout uh_layout(Arena& a, long long nb, long long np) {
  UhLayout l{};
  l.table.cap = (unsigned long long)std::max<long long>(2 * nb, 2);
  int r = 1;
  while (r < 31 && (1LL << r) - 1 < nb) ++r;  // nb <= 2^r - 1 (nb < 2^31)
  l.table.rbits = r;
  l.table.rmask = (1u << r) - 1;
  l.table.slot = a.take<unsigned>(l.table.cap);
  l.partner = a.take<int>(std::max<long long>(np, 1));
  l.bcnt = a.take<long long>((np + CB - 1) / CB + 1);
  l.total = a.take<long long>(1);
  return l;
}

// Queues the table's reset, build and probe, and the scan of the probe
// blocks' match counts (the total also into *count, a device address).
int uh_queue(const UhLayout& l, const int64_t* build0, const int64_t* build1, int64_t nb,
             const int64_t* probe0, const int64_t* probe1, int64_t np, int nkeys,
             long long* count, cudaStream_t st) {
  PF_CUDA(cudaMemsetAsync(l.table.slot, 0xff, l.table.cap * sizeof(unsigned), st));
  const unsigned nblk = blocks_for(np, CB);
  const long long* b0 = (const long long*)build0;
  const long long* b1 = (const long long*)(nkeys == 2 ? build1 : build0);
  const long long* p0 = (const long long*)probe0;
  const long long* p1 = (const long long*)(nkeys == 2 ? probe1 : probe0);
  if (nkeys == 2) {
    {
      PF_KERNEL("k_uh_build", st);
      k_uh_build<true><<<blocks_for(nb, T), T, 0, st>>>(b0, b1, nb, l.table);
    }
    {
      PF_KERNEL("k_uh_probe", st);
      k_uh_probe<true><<<nblk, CT, 0, st>>>(b0, b1, p0, p1, np, l.table, l.partner, l.bcnt);
    }
  } else {
    {
      PF_KERNEL("k_uh_build", st);
      k_uh_build<false><<<blocks_for(nb, T), T, 0, st>>>(b0, b1, nb, l.table);
    }
    {
      PF_KERNEL("k_uh_probe", st);
      k_uh_probe<false><<<nblk, CT, 0, st>>>(b0, b1, p0, p1, np, l.table, l.partner, l.bcnt);
    }
  }
  PF_LAUNCH("k_uh_build/k_uh_probe");
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.bcnt, nblk, l.total, count);
  }
  PF_LAUNCH("k_scan_counts");
  return PF_OK;
}

int uh_emit(const UhLayout& l, int64_t np, int64_t* build_idx, int64_t* probe_idx,
            cudaStream_t st) {
  {
    PF_KERNEL("k_uh_emit", st);
    k_uh_emit<<<blocks_for(np, CB), CT, 0, st>>>(l.partner, np, l.bcnt, (long long*)build_idx,
                                                 (long long*)probe_idx);
  }
  PF_LAUNCH("k_uh_emit");
  return PF_OK;
}

struct SaLayout {
  long long* table;
  long long* mn;
  long long* mx;
  unsigned char* keep;
  long long* bcnt;
  long long* dev;  // [0] kept rows, [1] bad
};

SaLayout sa_layout(Arena& a, long long nb, long long np, int op) {
  SaLayout l{};
  const uint64_t cap = pow2_at_least((uint64_t)std::max<long long>(2 * nb, 2));
  l.table = a.take<long long>(cap);
  const bool need_mn = op == PF_OP_NE || op == PF_OP_LT || op == PF_OP_LE;
  const bool need_mx = op == PF_OP_NE || op == PF_OP_GT || op == PF_OP_GE;
  l.mn = need_mn ? a.take<long long>(cap) : nullptr;
  l.mx = need_mx ? a.take<long long>(cap) : nullptr;
  l.keep = a.take<unsigned char>(std::max<long long>(np, 1));
  l.bcnt = a.take<long long>((np + CB - 1) / CB + 1);
  l.dev = a.take<long long>(2);
  return l;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" size_t pf_join_unique_hash_workspace(int64_t n_build, int64_t n_probe) {
  Arena a(nullptr, 0);
  uh_layout(a, n_build, n_probe);
  return a.used + 256;
}

extern "C" int pf_join_unique_hash(const int64_t* build0, const int64_t* build1, int64_t n_build,
                                   const int64_t* probe0, const int64_t* probe1, int64_t n_probe,
                                   int nkeys, int64_t* build_idx, int64_t* probe_idx,
                                   int64_t* host_out, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (nkeys != 1 && nkeys != 2) return fail(PF_EINVAL, "join_unique_hash: one or two keys, got %d", nkeys);
  if (n_build < 1 || n_probe < 1)
    return fail(PF_EINVAL, "join_unique_hash: unique hash needs rows on both sides");
  if (n_build > PF_JOIN_MAX_ROWS || n_probe > PF_JOIN_MAX_ROWS)
    return fail(PF_EINVAL, "join_unique_hash: a call takes at most %lld rows a side",
                (long long)PF_JOIN_MAX_ROWS);
  if (!build0 || !probe0 || (nkeys == 2 && (!build1 || !probe1)) || !build_idx || !probe_idx)
    return fail(PF_EINVAL, "join_unique_hash: null column");
  Arena a(workspace, workspace_bytes);
  UhLayout l = uh_layout(a, n_build, n_probe);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "join_unique_hash: workspace of %zu bytes, %zu needed",
                workspace_bytes, a.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  host_out[1] = 0;
  if (int rc = uh_queue(l, build0, build1, n_build, probe0, probe1, n_probe, nkeys, host_dev, st))
    return rc;
  cudaEvent_t ev;
  if (int rc = record_event(st, &ev)) return rc;
  if (int rc = uh_emit(l, n_probe, build_idx, probe_idx, st)) return rc;
  if (int rc = wait_event(ev)) return rc;
  return ok();
}

extern "C" size_t pf_join_semi_anti_workspace(int64_t n_build, int64_t n_probe, int op) {
  Arena a(nullptr, 0);
  sa_layout(a, n_build, n_probe, op);
  return a.used + 256;
}

extern "C" int pf_join_semi_anti(const int64_t* build_key, int64_t n_build,
                                 const int64_t* probe_key, int64_t n_probe,
                                 const int64_t* build_val, const int64_t* probe_val, int op,
                                 int anti, int64_t* out, int64_t* host_out, void* workspace,
                                 size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n_build < 1 || n_probe < 1)
    return fail(PF_EINVAL, "join_semi_anti: semi/anti needs rows on both sides");
  if (n_probe > PF_JOIN_MAX_ROWS || n_build > PF_JOIN_MAX_ROWS)
    return fail(PF_EINVAL, "join_semi_anti: a call takes at most %lld rows a side",
                (long long)PF_JOIN_MAX_ROWS);
  if (op < PF_OP_NONE || op > PF_OP_GE) return fail(PF_EINVAL, "join_semi_anti: unknown residual operator %d", op);
  if (op != PF_OP_NONE && (!build_val || !probe_val))
    return fail(PF_EINVAL, "join_semi_anti: a residual needs both value columns");
  Arena a(workspace, workspace_bytes);
  SaLayout l = sa_layout(a, n_build, n_probe, op);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "join_semi_anti: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  const uint64_t cap = pow2_at_least((uint64_t)std::max<long long>(2 * n_build, 2));
  const int logcap = log2_exact(cap);
  const unsigned fill_blocks = (unsigned)std::min<uint64_t>((cap + 255) / 256, 4096);
  {
    PF_KERNEL("k_fill_i64", st);
    k_fill_i64<<<fill_blocks, 256, 0, st>>>(l.table, EMPTY_KEY, (long long)cap);
  }
  if (l.mn) k_fill_i64<<<fill_blocks, 256, 0, st>>>(l.mn, LLONG_MAX, (long long)cap);
  if (l.mx) k_fill_i64<<<fill_blocks, 256, 0, st>>>(l.mx, LLONG_MIN, (long long)cap);
  host_out[0] = 0;
  host_out[1] = 0;  // the build below sets it through the alias
  {
    PF_KERNEL("k_set_build", st);
    k_set_build<<<blocks_for(n_build, T), T, 0, st>>>((const long long*)build_key,
                                                      (const long long*)build_val, n_build, l.table,
                                                      l.mn, l.mx, logcap, host_dev + 1);
  }
  PF_LAUNCH("k_set_build");
  const unsigned nblk = blocks_for(n_probe, CB);
  {
    PF_KERNEL("k_set_probe", st);
    k_set_probe<<<nblk, CT, 0, st>>>((const long long*)probe_key, (const long long*)probe_val,
                                     n_probe, l.table, l.mn, l.mx, logcap, op, anti != 0, l.keep,
                                     l.bcnt);
  }
  PF_LAUNCH("k_set_probe");
  {
    PF_KERNEL("k_scan_counts", st);
    k_scan_counts<<<1, 1024, 0, st>>>(l.bcnt, nblk, l.dev, host_dev);
  }
  PF_LAUNCH("k_scan_counts");
  cudaEvent_t ev;
  if (int rc = record_event(st, &ev)) return rc;
  {
    PF_KERNEL("k_keep_emit", st);
    k_keep_emit<<<nblk, CT, 0, st>>>(l.keep, n_probe, l.bcnt, (long long*)out);
  }
  PF_LAUNCH("k_keep_emit");
  if (int rc = wait_event(ev)) return rc;
  if (host_out[1] == 2) return fail(PF_EDEVICE, "join_semi_anti: the key set overflowed");
  return ok();
}

extern "C" size_t pf_join_expand_workspace(int64_t m) {
  Arena a(nullptr, 0);
  a.take<long long>(std::max<int64_t>(m, 1));           // incl
  a.take<long long>(1);                                 // total
  a.take<long long>(scan_scratch_elems(std::max<int64_t>(m, 1)));
  return a.used + 256;
}

namespace {
struct ExLayout {
  long long* incl;
  long long* total;
  long long* scratch;
};
ExLayout ex_layout(Arena& a, int64_t m) {
  ExLayout l{};
  l.incl = a.take<long long>(std::max<int64_t>(m, 1));
  l.total = a.take<long long>(1);
  l.scratch = a.take<long long>(scan_scratch_elems(std::max<int64_t>(m, 1)));
  return l;
}
}  // namespace

extern "C" int pf_join_expand_prepare(const int64_t* len, int64_t m, int64_t* host_out,
                                      void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (m < 0 || m > PF_JOIN_MAX_ROWS)
    return fail(PF_EINVAL, "join_expand: at most %lld probe rows", (long long)PF_JOIN_MAX_ROWS);
  Arena a(workspace, workspace_bytes);
  ExLayout l = ex_layout(a, m);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "join_expand: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  long long* host_dev = nullptr;
  if (int rc = host_alias(host_out, (void**)&host_dev)) return rc;
  if (m == 0) {
    host_out[0] = 0;
    return ok();
  }
  if (int rc = scan_i64((const long long*)len, l.incl, m, true, l.total, l.scratch, st)) return rc;
  {
    PF_KERNEL("k_copy_i64", st);
    k_copy_i64<<<1, 32, 0, st>>>(l.total, host_dev, 1);
  }
  PF_LAUNCH("k_copy_i64");
  if (int rc = wait_stream(st)) return rc;
  return ok();
}

extern "C" int pf_join_expand(const int64_t* sorted_ids, const int64_t* start, const int64_t* len,
                              int64_t m, int64_t n_pairs, int64_t* cs, int64_t* cr,
                              void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n_pairs <= 0 || m <= 0) return ok();
  Arena a(workspace, workspace_bytes);
  ExLayout l = ex_layout(a, m);
  if (!workspace || !a.fits())
    return fail(PF_ENOSPACE, "join_expand: workspace of %zu bytes, %zu needed", workspace_bytes,
                a.used);
  const long long threads = (n_pairs + EITEMS - 1) / EITEMS;
  {
    PF_KERNEL("k_expand", st);
    k_expand<<<blocks_for(threads, T), T, 0, st>>>((const long long*)sorted_ids,
                                                   (const long long*)start, (const long long*)len,
                                                   l.incl, m, n_pairs, (long long*)cs,
                                                   (long long*)cr);
  }
  PF_LAUNCH("k_expand");
  return ok();
}

// ---- unique hash join on static scratch (allocates nothing) -------------------
//
// pf_join_unique_hash with its scratch (hash table, per-row partners, per-block
// counts) in one file-scope device array instead of a caller's workspace, and
// its match count left on the device instead of a host wait.  The first call
// on a device, with that device current, looks the array's address up once
// (cudaGetSymbolAddress, which also loads this module on that device); later
// calls reuse it.  The array is shared: calls that overlap on one device, from
// two streams or two host threads, race on it.

namespace pf {
namespace {

__device__ __align__(256) unsigned char g_uh_static_scratch[PF_UH_STATIC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_uh_static_mu;
void* g_uh_static_ptr[MAX_DEVICES];

// This device's address of g_uh_static_scratch (looked up on first use).
int uh_static_scratch(void** out) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES)
    return fail(PF_EDEVICE, "join_unique_hash_static: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_uh_static_mu);
  if (!g_uh_static_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_uh_static_scratch);
    if (rc != cudaSuccess || !p)
      return fail(PF_ECUDA, "join_unique_hash_static: cudaGetSymbolAddress: %s",
                  cudaGetErrorString(rc));
    g_uh_static_ptr[dev] = p;
  }
  *out = g_uh_static_ptr[dev];
  return PF_OK;
}

}  // namespace
}  // namespace pf

extern "C" int pf_join_unique_hash_static(const int64_t* build0, const int64_t* build1,
                                          int64_t n_build, const int64_t* probe0,
                                          const int64_t* probe1, int64_t n_probe, int nkeys,
                                          int64_t* build_idx, int64_t* probe_idx,
                                          int64_t* match_count, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (nkeys != 1 && nkeys != 2)
    return fail(PF_EINVAL, "join_unique_hash_static: one or two keys, got %d", nkeys);
  if (n_build < 1 || n_probe < 1)
    return fail(PF_EINVAL, "join_unique_hash_static: unique hash needs rows on both sides");
  if (!build0 || !probe0 || (nkeys == 2 && (!build1 || !probe1)) || !build_idx || !probe_idx ||
      !match_count)
    return fail(PF_EINVAL, "join_unique_hash_static: null pointer");
  // the sizes must fit the fixed scratch (checked before anything is queued)
  if (n_build > PF_JOIN_MAX_ROWS || n_probe > PF_JOIN_MAX_ROWS)
    return fail(PF_EINVAL, "join_unique_hash_static: at most %lld rows a side",
                (long long)PF_JOIN_MAX_ROWS);
  Arena need(nullptr, 0);
  uh_layout(need, n_build, n_probe);
  if (need.used > (size_t)PF_UH_STATIC_SCRATCH_BYTES)
    return fail(PF_EINVAL,
                "join_unique_hash_static: %lld build x %lld probe rows need %zu bytes of "
                "scratch, the static scratch holds %zu (e.g. up to 524288 build with "
                "1048576 probe rows); use pf_join_unique_hash",
                (long long)n_build, (long long)n_probe, need.used,
                (size_t)PF_UH_STATIC_SCRATCH_BYTES);
  void* scratch = nullptr;
  if (int rc = uh_static_scratch(&scratch)) return rc;
  Arena a(scratch, PF_UH_STATIC_SCRATCH_BYTES);
  UhLayout l = uh_layout(a, n_build, n_probe);
  // the table starts empty (all ones) every call; partners, block counts and
  // the total are written in full before they are read
  if (int rc = uh_queue(l, build0, build1, n_build, probe0, probe1, n_probe, nkeys,
                        (long long*)match_count, st))
    return rc;
  if (int rc = uh_emit(l, n_probe, build_idx, probe_idx, st)) return rc;
  return ok();
}
