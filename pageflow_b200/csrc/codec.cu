// The PFC1 page encoder (host), and the paged workload's page builder: the
// probe table of the paged benchmark generated and encoded row group by row
// group on host threads, straight into compressed pages.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "codec.h"
#include "common.cuh"
#include "synth.h"

namespace pf {
namespace {

inline uint32_t bit_width(uint64_t r) { return r ? 64 - __builtin_clzll(r) : 0; }

void put(std::vector<uint8_t>& out, const void* p, size_t n) {
  const uint8_t* b = (const uint8_t*)p;
  out.insert(out.end(), b, b + n);
}

void align16(std::vector<uint8_t>& out) {
  while (out.size() % 16) out.push_back(0);
}

// A FOR or DELTA stream of v[0, n).
void encode_stream(const int64_t* v, uint32_t n, uint32_t scheme, std::vector<uint8_t>& out) {
  align16(out);
  const uint32_t nblk = (n + PFC_BLOCK - 1) / PFC_BLOCK;
  PfcStream sh{scheme, n, nblk, 0};
  put(out, &sh, sizeof(sh));
  std::vector<PfcBlock> blocks(nblk);
  std::vector<uint32_t> words;
  for (uint32_t k = 0; k < nblk; ++k) {
    const uint32_t j0 = k * PFC_BLOCK, cnt = std::min<uint32_t>(PFC_BLOCK, n - j0);
    // the block's terms: values (FOR) or differences after the first (DELTA)
    std::vector<uint64_t> t(cnt);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (uint32_t j = 0; j < cnt; ++j) {
      int64_t x;
      if (scheme == PFC_DELTA) x = j == 0 ? 0 : (int64_t)((uint64_t)v[j0 + j] - (uint64_t)v[j0 + j - 1]);
      else x = v[j0 + j];
      if (scheme == PFC_DELTA && j == 0) continue;
      lo = std::min(lo, x);
      hi = std::max(hi, x);
      t[j] = (uint64_t)x;
    }
    if (lo > hi) lo = hi = 0;  // a DELTA block of one value
    PfcBlock& b = blocks[k];
    std::memset(&b, 0, sizeof(b));
    b.base = lo;
    b.first = scheme == PFC_DELTA ? v[j0] : 0;
    b.bw = bit_width((uint64_t)hi - (uint64_t)lo);
    b.word_off = (uint32_t)words.size();
    const uint64_t nbits = (uint64_t)b.bw * cnt;
    const size_t base_w = words.size();
    words.resize(base_w + (size_t)((nbits + 31) / 32), 0u);
    if (b.bw) {
      for (uint32_t j = 0; j < cnt; ++j) {
        if (scheme == PFC_DELTA && j == 0) continue;
        const uint64_t d = t[j] - (uint64_t)lo;
        const uint64_t bit = (uint64_t)j * b.bw;
        uint32_t w = (uint32_t)(bit >> 5), sh2 = (uint32_t)(bit & 31);
        // up to 64 bits over up to three words
        words[base_w + w] |= (uint32_t)(d << sh2);
        uint32_t done = 32 - sh2;
        while (done < b.bw) {
          ++w;
          words[base_w + w] |= (uint32_t)(d >> done);
          done += 32;
        }
      }
    }
  }
  words.push_back(0u);
  words.push_back(0u);
  words.push_back(0u);
  put(out, blocks.data(), blocks.size() * sizeof(PfcBlock));
  put(out, words.data(), words.size() * sizeof(uint32_t));
  align16(out);
}

size_t stream_size(const int64_t* v, uint32_t n, uint32_t scheme) {
  std::vector<uint8_t> tmp;
  encode_stream(v, n, scheme, tmp);
  return tmp.size();
}

// Encodes one page of n values (as int64; esize the decoded width) with the
// smallest of RAW, FOR, DELTA and RLE (when its runs fit PFC_RLE_MAX_RUNS).
void encode_page(const int64_t* v, uint32_t n, int esize, std::vector<uint8_t>& out) {
  const size_t start = out.size();
  std::vector<int64_t> rv, re;
  for (uint32_t i = 0; i < n; ++i) {
    if (i == 0 || v[i] != v[i - 1]) {
      if (!rv.empty() && rv.size() > PFC_RLE_MAX_RUNS) break;
      rv.push_back(v[i]);
      re.push_back(0);
    }
    re.back() = i + 1;
  }
  const bool rle_ok = n > 0 && rv.size() <= PFC_RLE_MAX_RUNS && re.back() == (int64_t)n;
  const size_t raw = (size_t)esize * n + 16;
  const size_t s_for = stream_size(v, n, PFC_FOR);
  const size_t s_delta = stream_size(v, n, PFC_DELTA);
  size_t s_rle = SIZE_MAX;
  uint32_t rle_vs = PFC_FOR;
  if (rle_ok) {
    const size_t a = stream_size(rv.data(), (uint32_t)rv.size(), PFC_FOR);
    const size_t b = stream_size(rv.data(), (uint32_t)rv.size(), PFC_DELTA);
    rle_vs = b < a ? PFC_DELTA : PFC_FOR;
    s_rle = std::min(a, b) + stream_size(re.data(), (uint32_t)re.size(), PFC_DELTA);
  }
  uint8_t scheme = PFC_RAW;
  size_t best = raw;
  if (s_for < best) { best = s_for; scheme = PFC_FOR; }
  if (s_delta < best) { best = s_delta; scheme = PFC_DELTA; }
  if (s_rle < best) { best = s_rle; scheme = PFC_RLE; }
  PfcPage h;
  std::memset(&h, 0, sizeof(h));
  h.magic = PFC_MAGIC;
  h.scheme = scheme;
  h.esize = (uint8_t)esize;
  h.n = n;
  put(out, &h, sizeof(h));
  PfcPage* hp = nullptr;
  h.s0 = (uint32_t)(out.size() - start);
  if (scheme == PFC_RAW) {
    for (uint32_t i = 0; i < n; ++i) {
      if (esize == 8) put(out, &v[i], 8);
      else {
        const int32_t x = (int32_t)v[i];
        put(out, &x, 4);
      }
    }
    align16(out);
  } else if (scheme == PFC_RLE) {
    h.nruns = (uint32_t)rv.size();
    encode_stream(rv.data(), (uint32_t)rv.size(), rle_vs, out);
    h.s0 = (uint32_t)(sizeof(PfcPage));
    align16(out);
    h.s1 = (uint32_t)(out.size() - start);
    encode_stream(re.data(), (uint32_t)re.size(), PFC_DELTA, out);
  } else {
    encode_stream(v, n, scheme, out);
  }
  align16(out);
  h.bytes = (uint32_t)(out.size() - start);
  hp = (PfcPage*)(out.data() + start);
  std::memcpy(hp, &h, sizeof(h));
}

// The paged benchmark's probe table: 6 columns (fk int64, date int32, price
// int64, quantity int64, flag int32, status int32), generated per row r:
//   fk       1 + perm(rank), rank Zipf over n_build keys (the caller's table)
//   date     8035 + (r mod 2^20) * 2557 / 2^20: sorted within 2^20-row runs
//   price    90000 + range(u(seed,4,r), 10410001) cents
//   quantity 1 + range(u(seed,5,r), 50)
//   flag     range(u(seed,6,r), 3)
//   status   range(u(seed,7,r), 2)
struct PagedGen {
  uint64_t seed;
  int64_t n_rows, n_build;
  int rpp;  // rows per page (a row group)
  const int64_t* edges;
  const uint64_t* thr;
  int nbins;
};

constexpr int PAGED_COLS = 6;
constexpr int PAGED_ESIZE[PAGED_COLS] = {8, 4, 8, 8, 4, 4};

void gen_group(const PagedGen& g, int64_t grp, std::vector<uint8_t>& out,
               std::vector<int64_t>& sizes) {
  const int64_t r0 = grp * g.rpp, n = std::min<int64_t>(g.rpp, g.n_rows - r0);
  const pf_perm_t perm = pf_perm_make(g.seed, (uint64_t)g.n_build);
  std::vector<int64_t> col((size_t)n);
  for (int c = 0; c < PAGED_COLS; ++c) {
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t r = (uint64_t)(r0 + i);
      int64_t x = 0;
      switch (c) {
        case 0: {
          const uint64_t rank = pf_zipf_rank(pf_u(g.seed, 2, r), pf_u(g.seed, 3, r), g.nbins,
                                             g.edges, g.thr);
          x = (int64_t)(1 + pf_perm(&perm, rank));
          break;
        }
        case 1: x = 8035 + (int64_t)(((r & ((1u << 20) - 1)) * 2557) >> 20); break;
        case 2: x = 90000 + (int64_t)pf_range(pf_u(g.seed, 4, r), 10410001); break;
        case 3: x = 1 + (int64_t)pf_range(pf_u(g.seed, 5, r), 50); break;
        case 4: x = (int64_t)pf_range(pf_u(g.seed, 6, r), 3); break;
        default: x = (int64_t)pf_range(pf_u(g.seed, 7, r), 2); break;
      }
      col[(size_t)i] = x;
    }
    const size_t before = out.size();
    encode_page(col.data(), (uint32_t)n, PAGED_ESIZE[c], out);
    sizes.push_back((int64_t)(out.size() - before));
  }
}

struct PagedHandle {
  std::vector<std::vector<uint8_t>> parts;   // per worker
  std::vector<std::vector<int64_t>> sizes;   // per worker: page sizes in order
  std::vector<std::pair<int64_t, int64_t>> groups;  // per worker: [g0, g1)
  int64_t total = 0, n_groups = 0;
};

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" int64_t pf_page_encode(const void* values, int esize, int64_t n, void* out,
                                  int64_t capacity) {
  if ((esize != 4 && esize != 8) || n < 0 || n > (1LL << 30))
    return fail(PF_EINVAL, "page_encode: esize 4 or 8 and at most 2^30 values");
  std::vector<int64_t> v((size_t)n);
  for (int64_t i = 0; i < n; ++i)
    v[(size_t)i] = esize == 8 ? ((const int64_t*)values)[i] : ((const int32_t*)values)[i];
  std::vector<uint8_t> bytes;
  encode_page(v.data(), (uint32_t)n, esize, bytes);
  if ((int64_t)bytes.size() > capacity)
    return fail(PF_ENOSPACE, "page_encode: %zu bytes, capacity %lld", bytes.size(),
                (long long)capacity);
  std::memcpy(out, bytes.data(), bytes.size());
  ok();
  return (int64_t)bytes.size();
}

extern "C" int pf_paged_generate(uint64_t seed, int64_t n_rows, int rows_per_page,
                                 int64_t n_build, const int64_t* zipf_edges,
                                 const uint64_t* zipf_thr, int nbins, int threads,
                                 void** handle, int64_t* total_bytes) {
  if (n_rows < 1 || rows_per_page < PFC_BLOCK || rows_per_page % PFC_BLOCK || n_build < 1 ||
      nbins < 1)
    return fail(PF_EINVAL, "paged_generate: bad arguments");
  PagedGen g{seed, n_rows, n_build, rows_per_page, zipf_edges, zipf_thr, nbins};
  auto* h = new PagedHandle;
  h->n_groups = (n_rows + rows_per_page - 1) / rows_per_page;
  threads = std::max(1, std::min<int>(threads, (int)h->n_groups));
  h->parts.resize(threads);
  h->sizes.resize(threads);
  h->groups.resize(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const int64_t g0 = h->n_groups * t / threads, g1 = h->n_groups * (t + 1) / threads;
    h->groups[t] = {g0, g1};
    pool.emplace_back([&, t, g0, g1] {
      for (int64_t q = g0; q < g1; ++q) gen_group(g, q, h->parts[t], h->sizes[t]);
    });
  }
  for (auto& th : pool) th.join();
  for (auto& p : h->parts) h->total += (int64_t)p.size();
  *handle = h;
  *total_bytes = h->total;
  return ok();
}

// Copies the pages into dst (total_bytes) and each page's byte offset into
// directory[n_groups * 6] (row group major), then frees the handle.
extern "C" int pf_paged_fetch(void* handle, void* dst, int64_t* directory, int64_t* n_groups) {
  auto* h = (PagedHandle*)handle;
  if (!h) return fail(PF_EINVAL, "paged_fetch: null handle");
  int64_t off = 0, k = 0;
  for (size_t t = 0; t < h->parts.size(); ++t) {
    std::memcpy((uint8_t*)dst + off, h->parts[t].data(), h->parts[t].size());
    for (int64_t s : h->sizes[t]) {
      directory[k++] = off;
      off += s;
    }
  }
  *n_groups = h->n_groups;
  delete h;
  return ok();
}
