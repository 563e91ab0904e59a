/*
 * Seeded synthetic join workloads, counter-based so that the CUDA generator
 * (synth.cu) and the CPU one (the oracle's) produce the same columns from
 * (seed, stream, row) with no state.  Plain C99 + CUDA: PF_HD marks the
 * functions both compilers take.
 *
 *   u(seed, s, r)   splitmix64 finalizer (Steele, Lea, Flood 2014; constants
 *                   as published by Vigna) of the row under a per-stream key
 *   range(u, n)     floor(u * n / 2^64): uniform in [0, n) without modulo bias
 *                   beyond 2^-64
 *   perm(seed, N)   a bijection of [0, N): a 4-round Feistel network on the
 *                   smallest even bit width covering N, cycle-walked back into
 *                   [0, N); its inverse walks the rounds backwards
 *
 * Workload (the join + group-by the benchmark names):
 *   build row r:  key = 1 + perm(r)            (unique, a permutation of 1..N)
 *                 group = range(u(seed,1,r), G)
 *   probe row r:  miss = miss_per_10 > range(u(seed,2,r), 10)
 *                 fk = (miss ? N + 1 : 1) + range(u(seed,3,r), N)
 *                 price = 90000 + range(u(seed,4,r), 10410001)    cents
 *                 disc  = range(u(seed,5,r), 11)                  hundredths
 *
 * Serving workload (N ranked keys; a dimension of n keys holds the n most
 * referenced ranks, so smaller dimensions hold hotter keys):
 *   dimension row r:  key = 1 + perm(seed, N)(r), group = range(u(gseed,1,r), G)
 *   fact row r:       fk = 1 + perm(seed, N)(zipf rank(u(seed,2,r), u(seed,3,r)))
 *                     date = 8035 + range(u(seed,4,r), 2557)         days
 *                     value = 90000 + range(u(seed,5,r), 10410001)   cents
 */
#ifndef PF_SYNTH_H
#define PF_SYNTH_H

#include <stdint.h>

#ifdef __CUDACC__
#define PF_HD __host__ __device__ __forceinline__
#else
#define PF_HD static inline
#endif

PF_HD uint64_t pf_splitmix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* The per-(seed, stream) key, then the row through the finalizer. */
PF_HD uint64_t pf_u(uint64_t seed, uint32_t stream, uint64_t row) {
  uint64_t k = pf_splitmix(seed * 0x2545f4914f6cdd1dULL + stream);
  return pf_splitmix(k ^ (row * 0xd1b54a32d192ed03ULL));
}

PF_HD uint64_t pf_range(uint64_t u, uint64_t n) {
#ifdef __CUDA_ARCH__
  return __umul64hi(u, n);
#else
  return (uint64_t)(((unsigned __int128)u * n) >> 64);
#endif
}

/* Feistel permutation of [0, 2^(2*half)). */
typedef struct {
  uint64_t n;      /* the domain [0, n) */
  int half;        /* bits per Feistel half */
  uint64_t mask;   /* (1 << half) - 1 */
  uint64_t rk[4];  /* round keys */
} pf_perm_t;

PF_HD pf_perm_t pf_perm_make(uint64_t seed, uint64_t n) {
  pf_perm_t p;
  int bits = 1;
  while (bits < 62 && (1ULL << bits) < n) ++bits;
  p.n = n;
  p.half = (bits + 1) / 2;
  p.mask = (1ULL << p.half) - 1;
  for (int r = 0; r < 4; ++r) p.rk[r] = pf_splitmix(seed * 0x9e3779b97f4a7c15ULL + 0x1000 + r);
  return p;
}

PF_HD uint64_t pf_feistel_fwd(const pf_perm_t* p, uint64_t x) {
  uint64_t l = x >> p->half, r = x & p->mask;
  for (int i = 0; i < 4; ++i) {
    uint64_t nl = r;
    r = l ^ (pf_splitmix(p->rk[i] ^ r) & p->mask);
    l = nl;
  }
  return (l << p->half) | r;
}

PF_HD uint64_t pf_feistel_inv(const pf_perm_t* p, uint64_t y) {
  uint64_t l = y >> p->half, r = y & p->mask;
  for (int i = 3; i >= 0; --i) {
    uint64_t nr = l;
    l = r ^ (pf_splitmix(p->rk[i] ^ l) & p->mask);
    r = nr;
  }
  return (l << p->half) | r;
}

/* Cycle walking: the first image inside [0, n).  x < n lies on its own
 * cycle, so the walk ends within that cycle's length. */
PF_HD uint64_t pf_perm(const pf_perm_t* p, uint64_t x) {
  uint64_t y = pf_feistel_fwd(p, x);
  while (y >= p->n) y = pf_feistel_fwd(p, y);
  return y;
}

PF_HD uint64_t pf_perm_inv(const pf_perm_t* p, uint64_t y) {
  uint64_t x = pf_feistel_inv(p, y);
  while (x >= p->n) x = pf_feistel_inv(p, x);
  return x;
}

/* Misses per ten probe rows of each workload config: config 0 (250K x 1M)
 * draws every FK from the build keys, config 1 (150M x 600M) one in ten from
 * outside them. */
PF_HD int pf_cfg_miss_per_10(int config) { return config == 0 ? 0 : 1; }

PF_HD void pf_gen_build_row(uint64_t seed, uint64_t n_build, uint64_t n_groups,
                            const pf_perm_t* perm, uint64_t r, int64_t* key, int32_t* group) {
  *key = (int64_t)(1 + pf_perm(perm, r));
  *group = (int32_t)pf_range(pf_u(seed, 1, r), n_groups);
  (void)n_build;
}

PF_HD void pf_gen_probe_row(uint64_t seed, uint64_t n_build, int miss_per_10, uint64_t r,
                            int64_t* fk, int64_t* price, int64_t* disc) {
  int miss = (uint64_t)miss_per_10 > pf_range(pf_u(seed, 2, r), 10);
  *fk = (int64_t)((miss ? n_build + 1 : 1) + pf_range(pf_u(seed, 3, r), n_build));
  *price = (int64_t)(90000 + pf_range(pf_u(seed, 4, r), 10410001));
  *disc = (int64_t)pf_range(pf_u(seed, 5, r), 11);
}

/*
 * The batching workload's probe rows (one instance, its own seed): the FK's
 * rank among the instance's n_build keys follows a Zipf law, sampled with a
 * table the host computes once per instance: nbins bins of ranks
 * [edges[b], edges[b+1]) and cumulative probabilities thr[b] (scaled to
 * 2^64, thr[nbins-1] = 2^64 - 1); the bin is the first whose threshold
 * exceeds u, the rank uniform inside it.  Uniform FKs are one bin.  Integer
 * only, so the CPU and the GPU draw the same rows.
 *   fk = 1 + perm(rank)          (hot ranks land on scattered keys)
 *   value = range(u(seed,5,r), 10^7)   cents
 */
PF_HD uint64_t pf_zipf_rank(uint64_t u_bin, uint64_t u_in, int nbins, const int64_t* edges,
                            const uint64_t* thr) {
  int lo = 0, hi = nbins - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (u_bin < thr[mid]) hi = mid;
    else lo = mid + 1;
  }
  const uint64_t width = (uint64_t)(edges[lo + 1] - edges[lo]);
  return (uint64_t)edges[lo] + pf_range(u_in, width);
}

PF_HD void pf_gen_batch_probe_row(uint64_t seed, const pf_perm_t* perm, int nbins,
                                  const int64_t* edges, const uint64_t* thr, uint64_t r,
                                  int64_t* fk, int64_t* value) {
  const uint64_t rank = pf_zipf_rank(pf_u(seed, 3, r), pf_u(seed, 4, r), nbins, edges, thr);
  *fk = (int64_t)(1 + pf_perm(perm, rank));
  *value = (int64_t)pf_range(pf_u(seed, 5, r), 10000000);
}

PF_HD void pf_gen_serve_dim_row(uint64_t gseed, const pf_perm_t* perm, uint64_t n_groups,
                                uint64_t r, int64_t* key, int32_t* group) {
  *key = (int64_t)(1 + pf_perm(perm, r));
  *group = (int32_t)pf_range(pf_u(gseed, 1, r), n_groups);
}

PF_HD void pf_gen_serve_fact_row(uint64_t seed, const pf_perm_t* perm, int nbins,
                                 const int64_t* edges, const uint64_t* thr, uint64_t r,
                                 int64_t* fk, int32_t* date, int64_t* value) {
  const uint64_t rank = pf_zipf_rank(pf_u(seed, 2, r), pf_u(seed, 3, r), nbins, edges, thr);
  *fk = (int64_t)(1 + pf_perm(perm, rank));
  *date = (int32_t)(8035 + pf_range(pf_u(seed, 4, r), 2557));
  *value = (int64_t)(90000 + pf_range(pf_u(seed, 5, r), 10410001));
}

#endif /* PF_SYNTH_H */
