/*
 * ORACLE — test infrastructure only.  A plain-C restatement of PageFlow's
 * CPU-visible semantics for the relational hot path, used by tests/ and by
 * bench.py's CPU baseline as the checker and the reference arm; never by the
 * product (pageflow_b200/), which runs on the GPU or fails.
 *
 * Pinned against golden vectors generated from the reference's own Python
 * code (tests/golden/make_golden.py, run where the reference is importable):
 * mix64 / bucket ids, the padded partition layout, the partition-count rule,
 * the slab and sorted-run merge vectors, and the config-0 join + group-by
 * result of the reference's KeyedAggregate.pass1 + reduce_tick_slice.
 *
 * Functions and the reference lines they follow:
 *   or_mix64            operators/kernels/kernel_utils.cuh:18-22; tests/mix64.py:12-21
 *   or_bucket           operators/aggregate.py:107-116; tests/mix64.py:30-36
 *   or_partition_order  tests/operators/test_partition_sort.py:106-118 (mask ->
 *                       mix64 bucket -> stable sort by bucket -> per-bucket split)
 *   or_join_unique      operators/hashjoin.py:380-441 (_sort_search_pairs: per
 *                       bucket sort of the build keys, searchsorted of each probe
 *                       key; pairs in probe-row order) for a unique build tuple,
 *                       operators/join_core.py:97-113
 *   or_semi_anti        tests/operators/test_join_core.py:93-101 (a probe row is
 *                       kept when some build row has its key and passes
 *                       build.v OP probe.v; anti negates), ascending
 *   or_join_aggregate   uvm/join.py:98-225 then uvm/aggregate.py:147-212: the
 *                       inner join, then SUM / COUNT per group; SUM follows
 *                       operators/operator_utils.py:389-398 (float64 bincount,
 *                       rounded to int64), exact while every partial < 2^53,
 *                       which the oracle checks and reports
 *   or_expected_groups  the same join + group-by computed from the generator
 *                       alone (the inverse of the build-key permutation gives
 *                       each FK's build row), for full-size checks
 *   or_gen_build/probe  the CPU twin of the CUDA generator (synth.h)
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../pageflow_b200/csrc/synth.h"

/* ---- mix64 and buckets ---------------------------------------------------- */

static inline uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

static inline int log2i(int64_t b) {
  int l = 0;
  while ((1LL << l) < b) ++l;
  return l;
}

static inline int bucket(int64_t key, int logb) {
  return logb ? (int)(mix64((uint64_t)key) >> (64 - logb)) : 0;
}

void or_mix64(const int64_t* in, uint64_t* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) out[i] = mix64((uint64_t)in[i]);
}

void or_bucket(const int64_t* keys, int64_t n, int B, int32_t* out) {
  const int lb = log2i(B);
  for (int64_t i = 0; i < n; ++i) out[i] = bucket(keys[i], lb);
}

/* Stable partition of n keys into B buckets: counts[B] and order[n], the rows
 * sorted by bucket, source order kept inside a bucket (a counting sort, which
 * is the stable sort of the reference test). */
int or_partition_order(const int64_t* keys, int64_t n, int B, int64_t* counts, int64_t* order) {
  if (B < 1 || (B & (B - 1))) return -1;
  const int lb = log2i(B);
  int32_t* bk = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  int64_t* at = (int64_t*)calloc((size_t)B, sizeof(int64_t));
  if (!bk || !at) {
    free(bk);
    free(at);
    return -2;
  }
  memset(counts, 0, sizeof(int64_t) * B);
  for (int64_t i = 0; i < n; ++i) {
    bk[i] = bucket(keys[i], lb);
    counts[bk[i]]++;
  }
  int64_t s = 0;
  for (int b = 0; b < B; ++b) {
    at[b] = s;
    s += counts[b];
  }
  for (int64_t i = 0; i < n; ++i) order[at[bk[i]]++] = i;
  free(bk);
  free(at);
  return 0;
}

/* ---- sort helpers --------------------------------------------------------- */

typedef struct {
  int64_t k0, k1, v;
  int64_t row;
} rec_t;

static int cmp_rec(const void* a, const void* b) {
  const rec_t* x = (const rec_t*)a;
  const rec_t* y = (const rec_t*)b;
  if (x->k0 != y->k0) return x->k0 < y->k0 ? -1 : 1;
  if (x->k1 != y->k1) return x->k1 < y->k1 ? -1 : 1;
  if (x->row != y->row) return x->row < y->row ? -1 : 1;
  return 0;
}

/* First index in r[0,n) whose (k0,k1) >= (a,b). */
static int64_t lower(const rec_t* r, int64_t n, int64_t a, int64_t b) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (r[mid].k0 < a || (r[mid].k0 == a && r[mid].k1 < b)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

/* ---- unique-build inner join --------------------------------------------- */

/* (build_idx, probe_idx) of every probe row whose tuple is in the build, in
 * probe-row order; returns their number (or < 0 on allocation failure).  A
 * probe row takes the first build row (in build order) with its tuple. */
int64_t or_join_unique(const int64_t* b0, const int64_t* b1, int64_t nb, const int64_t* p0,
                       const int64_t* p1, int64_t np, int nkeys, int64_t* build_idx,
                       int64_t* probe_idx) {
  rec_t* r = (rec_t*)malloc(sizeof(rec_t) * (nb > 0 ? nb : 1));
  if (!r) return -1;
  for (int64_t i = 0; i < nb; ++i) {
    r[i].k0 = b0[i];
    r[i].k1 = nkeys == 2 ? b1[i] : 0;
    r[i].v = 0;
    r[i].row = i;
  }
  qsort(r, (size_t)nb, sizeof(rec_t), cmp_rec);
  int64_t m = 0;
  for (int64_t i = 0; i < np; ++i) {
    const int64_t a = p0[i], b = nkeys == 2 ? p1[i] : 0;
    const int64_t j = lower(r, nb, a, b);
    if (j < nb && r[j].k0 == a && r[j].k1 == b) {
      build_idx[m] = r[j].row;
      probe_idx[m] = i;
      ++m;
    }
  }
  free(r);
  return m;
}

/* ---- semi / anti ----------------------------------------------------------- */

/* op: 0 none, 1 <>, 2 <, 3 <=, 4 >, 5 >= (build.v OP probe.v). */
int64_t or_semi_anti(const int64_t* bk, const int64_t* bv, int64_t nb, const int64_t* pk,
                     const int64_t* pv, int64_t np, int op, int anti, int64_t* out) {
  rec_t* r = (rec_t*)malloc(sizeof(rec_t) * (nb > 0 ? nb : 1));
  if (!r) return -1;
  for (int64_t i = 0; i < nb; ++i) {
    r[i].k0 = bk[i];
    r[i].k1 = 0;
    r[i].v = bv ? bv[i] : 0;
    r[i].row = i;
  }
  qsort(r, (size_t)nb, sizeof(rec_t), cmp_rec);
  int64_t m = 0;
  for (int64_t i = 0; i < np; ++i) {
    int64_t j = lower(r, nb, pk[i], 0);
    int hit = 0;
    for (; j < nb && r[j].k0 == pk[i] && !hit; ++j) {
      if (op == 0) {
        hit = 1;
      } else {
        const int64_t a = r[j].v, b = pv[i];
        switch (op) {
          case 1: hit = a != b; break;
          case 2: hit = a < b; break;
          case 3: hit = a <= b; break;
          case 4: hit = a > b; break;
          default: hit = a >= b; break;
        }
      }
    }
    if (hit != (anti != 0)) out[m++] = i;
  }
  free(r);
  return m;
}

/* ---- join + group-by ---------------------------------------------------------- */

typedef struct {
  const int64_t *bkey, *pfk, *pprice, *pdisc;
  const int32_t* bgrp;
  int64_t scale, gmin, ngroups;
  const int64_t *bstart, *pstart; /* per bucket row ranges of the partitioned sides */
  const int64_t *border, *porder;
  int B, b0, b1;                  /* this worker's buckets */
  int64_t* sum;                   /* private [ngroups] */
  int64_t* count;                 /* private [ngroups] */
  int64_t matched;
  int rc;
} jw_t;

static void* join_worker(void* arg) {
  jw_t* w = (jw_t*)arg;
  int64_t cap = 0;
  rec_t* r = NULL;
  for (int b = w->b0; b < w->b1; ++b) {
    const int64_t n = w->bstart[b + 1] - w->bstart[b];
    if (n > cap) {
      free(r);
      cap = n;
      r = (rec_t*)malloc(sizeof(rec_t) * (size_t)cap);
      if (!r) {
        w->rc = -1;
        return NULL;
      }
    }
    for (int64_t j = 0; j < n; ++j) {
      const int64_t row = w->border[w->bstart[b] + j];
      r[j].k0 = w->bkey[row];
      r[j].k1 = 0;
      r[j].v = w->bgrp[row];
      r[j].row = row;
    }
    qsort(r, (size_t)n, sizeof(rec_t), cmp_rec);
    for (int64_t q = w->pstart[b]; q < w->pstart[b + 1]; ++q) {
      const int64_t row = w->porder[q];
      const int64_t k = w->pfk[row];
      const int64_t j = lower(r, n, k, 0);
      if (j < n && r[j].k0 == k) {
        const int64_t g = r[j].v - w->gmin;
        w->matched++;
        if (g < 0 || g >= w->ngroups) continue;
        const int64_t v = w->pdisc ? (int64_t)((uint64_t)w->pprice[row] *
                                               (uint64_t)(w->scale - w->pdisc[row]))
                                   : w->pprice[row];
        w->sum[g] = (int64_t)((uint64_t)w->sum[g] + (uint64_t)v);
        w->count[g]++;
      }
    }
  }
  free(r);
  return NULL;
}

/* SELECT group, SUM(price * (scale - disc)), COUNT(*) over the unique-build
 * join, into dense sum / count arrays over [gmin, gmin + ngroups).  Both sides
 * are partitioned into B buckets by mix64 (the reference's layout), buckets
 * are joined by sort + binary search on `threads` threads.  Returns the
 * matched probe rows; *max_abs gets the largest |group sum| (the reference's
 * float64 SUM is exact below 2^53).  < 0 on failure. */
int64_t or_join_aggregate(const int64_t* bkey, const int32_t* bgrp, int64_t nb,
                          const int64_t* pfk, const int64_t* pprice, const int64_t* pdisc,
                          int64_t scale, int64_t np, int64_t gmin, int64_t ngroups, int B,
                          int threads, int64_t* sum, int64_t* count, uint64_t* max_abs) {
  if (threads < 1) threads = 1;
  if (B < 1) B = 1;
  int64_t* bc = (int64_t*)malloc(sizeof(int64_t) * B);
  int64_t* pc = (int64_t*)malloc(sizeof(int64_t) * B);
  int64_t* bs = (int64_t*)malloc(sizeof(int64_t) * (B + 1));
  int64_t* ps = (int64_t*)malloc(sizeof(int64_t) * (B + 1));
  int64_t* bo = (int64_t*)malloc(sizeof(int64_t) * (nb > 0 ? nb : 1));
  int64_t* po = (int64_t*)malloc(sizeof(int64_t) * (np > 0 ? np : 1));
  jw_t* ws = (jw_t*)calloc((size_t)threads, sizeof(jw_t));
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  int64_t result = -1;
  if (!bc || !pc || !bs || !ps || !bo || !po || !ws || !th) goto done;
  if (or_partition_order(bkey, nb, B, bc, bo) || or_partition_order(pfk, np, B, pc, po)) goto done;
  bs[0] = ps[0] = 0;
  for (int b = 0; b < B; ++b) {
    bs[b + 1] = bs[b] + bc[b];
    ps[b + 1] = ps[b] + pc[b];
  }
  for (int t = 0; t < threads; ++t) {
    jw_t* w = &ws[t];
    w->bkey = bkey;
    w->bgrp = bgrp;
    w->pfk = pfk;
    w->pprice = pprice;
    w->pdisc = pdisc;
    w->scale = scale;
    w->gmin = gmin;
    w->ngroups = ngroups;
    w->bstart = bs;
    w->pstart = ps;
    w->border = bo;
    w->porder = po;
    w->B = B;
    w->b0 = (int)((int64_t)B * t / threads);
    w->b1 = (int)((int64_t)B * (t + 1) / threads);
    w->sum = (int64_t*)calloc((size_t)ngroups, sizeof(int64_t));
    w->count = (int64_t*)calloc((size_t)ngroups, sizeof(int64_t));
    if (!w->sum || !w->count) goto done;
  }
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, join_worker, &ws[t]);
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  memset(sum, 0, sizeof(int64_t) * ngroups);
  memset(count, 0, sizeof(int64_t) * ngroups);
  int64_t matched = 0;
  for (int t = 0; t < threads; ++t) {
    if (ws[t].rc) goto done;
    matched += ws[t].matched;
    for (int64_t g = 0; g < ngroups; ++g) {
      sum[g] = (int64_t)((uint64_t)sum[g] + (uint64_t)ws[t].sum[g]);
      count[g] += ws[t].count[g];
    }
  }
  uint64_t mx = 0;
  for (int64_t g = 0; g < ngroups; ++g) {
    const uint64_t a = sum[g] < 0 ? (uint64_t)(-(sum[g] + 1)) + 1 : (uint64_t)sum[g];
    if (a > mx) mx = a;
  }
  if (max_abs) *max_abs = mx;
  result = matched;
done:
  if (ws)
    for (int t = 0; t < threads; ++t) {
      free(ws[t].sum);
      free(ws[t].count);
    }
  free(bc);
  free(pc);
  free(bs);
  free(ps);
  free(bo);
  free(po);
  free(ws);
  free(th);
  return result;
}

/* ---- generator --------------------------------------------------------------- */

void or_gen_build(uint64_t seed, int64_t n_build, int64_t n_groups, int64_t lo, int64_t rows,
                  int64_t* key, int32_t* group) {
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  for (int64_t i = 0; i < rows; ++i)
    pf_gen_build_row(seed, (uint64_t)n_build, (uint64_t)n_groups, &perm, (uint64_t)(lo + i),
                     &key[i], &group[i]);
}

void or_gen_probe(int config, uint64_t seed, int64_t n_build, int64_t lo, int64_t rows,
                  int64_t* fk, int64_t* price, int64_t* disc) {
  const int miss = pf_cfg_miss_per_10(config);
  for (int64_t i = 0; i < rows; ++i)
    pf_gen_probe_row(seed, (uint64_t)n_build, miss, (uint64_t)(lo + i), &fk[i], &price[i],
                     &disc[i]);
}

/* The CPU twin of one batching instance's probe rows (synth.h). */
void or_gen_batch_probe(uint64_t seed, int64_t n_build, int64_t lo, int64_t rows, int nbins,
                        const int64_t* edges, const uint64_t* thr, int64_t* fk, int64_t* value) {
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  for (int64_t i = 0; i < rows; ++i)
    pf_gen_batch_probe_row(seed, &perm, nbins, edges, thr, (uint64_t)(lo + i), &fk[i], &value[i]);
}

typedef struct {
  int config;
  uint64_t seed;
  int64_t n_build, n_groups, lo, hi;
  int64_t scale;
  const pf_perm_t* perm;
  int64_t *sum, *count, matched;
} ew_t;

static void* expect_worker(void* arg) {
  ew_t* w = (ew_t*)arg;
  const int miss = pf_cfg_miss_per_10(w->config);
  for (int64_t r = w->lo; r < w->hi; ++r) {
    int64_t fk, price, disc;
    pf_gen_probe_row(w->seed, (uint64_t)w->n_build, miss, (uint64_t)r, &fk, &price, &disc);
    if (fk < 1 || fk > w->n_build) continue;
    const uint64_t brow = pf_perm_inv(w->perm, (uint64_t)(fk - 1));
    const int64_t g = (int64_t)pf_range(pf_u(w->seed, 1, brow), (uint64_t)w->n_groups);
    w->sum[g] = (int64_t)((uint64_t)w->sum[g] + (uint64_t)price * (uint64_t)(w->scale - disc));
    w->count[g]++;
    w->matched++;
  }
  return NULL;
}

/* The workload's exact per-group SUM(price * (scale - disc)) and COUNT over
 * probe rows [lo, lo + rows), from the generator: FK f matches build row
 * perm^-1(f - 1), whose group the generator gives.  Returns matched rows. */
int64_t or_expected_groups(int config, uint64_t seed, int64_t n_build, int64_t n_groups,
                           int64_t scale, int64_t lo, int64_t rows, int threads, int64_t* sum,
                           int64_t* count) {
  if (threads < 1) threads = 1;
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  ew_t* ws = (ew_t*)calloc((size_t)threads, sizeof(ew_t));
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  if (!ws || !th) return -1;
  for (int t = 0; t < threads; ++t) {
    ws[t].config = config;
    ws[t].seed = seed;
    ws[t].n_build = n_build;
    ws[t].n_groups = n_groups;
    ws[t].scale = scale;
    ws[t].perm = &perm;
    ws[t].lo = lo + rows * t / threads;
    ws[t].hi = lo + rows * (t + 1) / threads;
    ws[t].sum = (int64_t*)calloc((size_t)n_groups, sizeof(int64_t));
    ws[t].count = (int64_t*)calloc((size_t)n_groups, sizeof(int64_t));
    if (!ws[t].sum || !ws[t].count) return -1;
  }
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, expect_worker, &ws[t]);
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  memset(sum, 0, sizeof(int64_t) * n_groups);
  memset(count, 0, sizeof(int64_t) * n_groups);
  int64_t matched = 0;
  for (int t = 0; t < threads; ++t) {
    for (int64_t g = 0; g < n_groups; ++g) {
      sum[g] = (int64_t)((uint64_t)sum[g] + (uint64_t)ws[t].sum[g]);
      count[g] += ws[t].count[g];
    }
    matched += ws[t].matched;
    free(ws[t].sum);
    free(ws[t].count);
  }
  free(ws);
  free(th);
  return matched;
}

/* ---- compressed pages ------------------------------------------------------ */
/*
 * A PFC1 page decoder restated from the format's definition (the page header,
 * stream header and block table of pageflow_b200/csrc/codec.h), independent of
 * the product's decoder: fields are read byte by byte and bit fields bit by
 * bit.  It stands for the decode half of the reference's codec binding
 * (compression/nvcomp_manager.cu:679 mgr_decompress of the CASCADED codec
 * configured at :162-173): a page decodes to exactly the values encoded.
 */
static uint64_t rd_u(const uint8_t* p, int bytes) {
  uint64_t x = 0;
  for (int i = 0; i < bytes; ++i) x |= (uint64_t)p[i] << (8 * i);
  return x;
}

static uint64_t rd_bits(const uint8_t* words, uint64_t j, uint32_t bw) {
  uint64_t v = 0;
  for (uint32_t b = 0; b < bw; ++b) {
    const uint64_t bit = j * bw + b;
    v |= (uint64_t)((words[bit >> 3] >> (bit & 7)) & 1u) << b;
  }
  return v;
}

/* One FOR / DELTA stream at byte offset off of a page of `bytes`; n values
 * expected.  Returns 0, or -1 when the stream is malformed. */
static int decode_stream(const uint8_t* page, uint64_t bytes, uint64_t off, uint64_t n,
                         int64_t* out) {
  if (off + 16 > bytes) return -1;
  const uint32_t scheme = (uint32_t)rd_u(page + off, 4);
  const uint64_t sn = rd_u(page + off + 4, 4), nblk = rd_u(page + off + 8, 4);
  if ((scheme != 1 && scheme != 2) || sn != n || nblk != (n + 1023) / 1024) return -1;
  const uint64_t tab = off + 16, words = tab + 32 * nblk;
  if (words > bytes) return -1;
  for (uint64_t k = 0; k < nblk; ++k) {
    const uint8_t* b = page + tab + 32 * k;
    const uint64_t base = rd_u(b, 8), first = rd_u(b + 8, 8);
    const uint64_t woff = rd_u(b + 16, 4), bw = rd_u(b + 20, 4);
    if (bw > 64) return -1;
    const uint64_t cnt = n - 1024 * k < 1024 ? n - 1024 * k : 1024;
    if (words + 4 * woff + (bw * cnt + 7) / 8 > bytes) return -1;
    uint64_t prev = 0;
    for (uint64_t j = 0; j < cnt; ++j) {
      const uint64_t field = base + rd_bits(page + words + 4 * woff, j, (uint32_t)bw);
      uint64_t v;
      if (scheme == 1) v = field;
      else v = j == 0 ? first : prev + field;
      out[1024 * k + j] = (int64_t)v;
      prev = v;
    }
  }
  return 0;
}

/* Decodes the page at page[0, bytes) into out[0, capacity) as int64 (int32
 * columns sign-extended).  Returns the page's rows, or -1 for a malformed
 * page, -2 when capacity is short. */
int64_t or_page_decode(const uint8_t* page, int64_t bytes, int64_t* out, int64_t capacity) {
  if (bytes < 64 || rd_u(page, 4) != 0x31434650u) return -1;
  const int scheme = page[4], esize = page[5];
  const uint64_t n = rd_u(page + 8, 4), nruns = rd_u(page + 12, 4);
  const uint64_t s0 = rd_u(page + 16, 4), s1 = rd_u(page + 20, 4), pb = rd_u(page + 24, 4);
  if ((esize != 4 && esize != 8) || pb > (uint64_t)bytes || pb % 16) return -1;
  if ((int64_t)n > capacity) return -2;
  if (scheme == 0) {
    if (s0 + n * (uint64_t)esize > pb) return -1;
    for (uint64_t i = 0; i < n; ++i) {
      const uint64_t x = rd_u(page + s0 + i * esize, esize);
      out[i] = esize == 8 ? (int64_t)x : (int64_t)(int32_t)(uint32_t)x;
    }
    return (int64_t)n;
  }
  if (scheme == 1 || scheme == 2) {
    if (decode_stream(page, pb, s0, n, out)) return -1;
  } else if (scheme == 3) {
    if (nruns == 0 || nruns > 4096 || nruns > n) return -1;
    int64_t* v = (int64_t*)malloc(sizeof(int64_t) * nruns);
    int64_t* e = (int64_t*)malloc(sizeof(int64_t) * nruns);
    int bad = !v || !e || decode_stream(page, pb, s0, nruns, v) ||
              decode_stream(page, pb, s1, nruns, e);
    int64_t row = 0;
    for (uint64_t r = 0; !bad && r < nruns; ++r) {
      if (e[r] <= row || e[r] > (int64_t)n) {
        bad = 1;
        break;
      }
      for (; row < e[r]; ++row) out[row] = v[r];
    }
    if (!bad && row != (int64_t)n) bad = 1;
    free(v);
    free(e);
    if (bad) return -1;
  } else {
    return -1;
  }
  if (esize == 4)
    for (uint64_t i = 0; i < n; ++i) out[i] = (int64_t)(int32_t)(uint32_t)(uint64_t)out[i];
  return (int64_t)n;
}

/* The CPU twin of the paged workload's probe table (pageflow_b200/csrc/
 * codec.cu), rows [lo, lo + rows) of its 6 columns as int64: fk (Zipf rank
 * over n_build keys through the key permutation), date (sorted within
 * 2^20-row runs over [8035, 10591]), price, quantity, flag, status. */
void or_gen_paged(uint64_t seed, int64_t n_build, int nbins, const int64_t* edges,
                  const uint64_t* thr, int64_t lo, int64_t rows, int64_t* fk, int64_t* date,
                  int64_t* price, int64_t* qty, int64_t* flag, int64_t* status) {
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_build);
  for (int64_t i = 0; i < rows; ++i) {
    const uint64_t r = (uint64_t)(lo + i);
    const uint64_t rank = pf_zipf_rank(pf_u(seed, 2, r), pf_u(seed, 3, r), nbins, edges, thr);
    fk[i] = (int64_t)(1 + pf_perm(&perm, rank));
    date[i] = 8035 + (int64_t)(((r % (1u << 20)) * 2557u) / (1u << 20));
    price[i] = 90000 + (int64_t)pf_range(pf_u(seed, 4, r), 10410001);
    qty[i] = 1 + (int64_t)pf_range(pf_u(seed, 5, r), 50);
    flag[i] = (int64_t)pf_range(pf_u(seed, 6, r), 3);
    status[i] = (int64_t)pf_range(pf_u(seed, 7, r), 2);
  }
}

/* The CPU twin of the serving workload's generator (synth.h): dimension rows
 * [lo, lo + rows) and fact rows [lo, lo + rows). */
void or_gen_serve_dim(uint64_t seed, int64_t n_ranks, uint64_t group_seed, int64_t n_groups,
                      int64_t lo, int64_t rows, int64_t* key, int32_t* group) {
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_ranks);
  for (int64_t i = 0; i < rows; ++i)
    pf_gen_serve_dim_row(group_seed, &perm, (uint64_t)n_groups, (uint64_t)(lo + i), &key[i],
                         &group[i]);
}

void or_gen_serve_fact(uint64_t seed, int64_t n_ranks, int nbins, const int64_t* edges,
                       const uint64_t* thr, int64_t lo, int64_t rows, int64_t* fk,
                       int32_t* date, int64_t* value) {
  const pf_perm_t perm = pf_perm_make(seed, (uint64_t)n_ranks);
  for (int64_t i = 0; i < rows; ++i)
    pf_gen_serve_fact_row(seed, &perm, nbins, edges, thr, (uint64_t)(lo + i), &fk[i], &date[i],
                          &value[i]);
}
