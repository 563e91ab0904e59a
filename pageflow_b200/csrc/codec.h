/*
 * PFC1: the cascaded integer page format of pageflow_b200 (plain C99 + CUDA).
 *
 * A page holds n values of one int32 or int64 column (esize 4 or 8).  Its
 * value stream is encoded by one scheme:
 *   FOR        frame of reference: per mini-block of PFC_BLOCK values, the
 *              minimum (base) and the bit width of (value - base); the
 *              differences bit-packed LSB first
 *   DELTA      the same over the differences of consecutive values, each
 *              block also storing its first value (blocks decode alone)
 *   RLE        run-length: the runs' values as a FOR or DELTA stream and the
 *              runs' exclusive end rows as a DELTA stream (ends increase)
 *   RAW        the values as they are
 * RLE + DELTA + bit packing cascade as in the reference's codec configuration
 * (nvCOMP CASCADED with RLE, delta and bit packing, compression/
 * nvcomp_manager.cu:162-173), in a layout of our own: every mini-block carries
 * its base, first value and the word offset of its bits, so any block decodes
 * without the ones before it (a GPU thread per value, a block-wide scan for
 * DELTA).
 *
 * Layout (little endian, every section 16-byte aligned):
 *   PfcPage header (64 B)
 *   stream 0 (values, or the runs' values)      at header.s0
 *   stream 1 (RLE only: the runs' ends)         at header.s1
 * A stream: PfcStream (16 B), PfcBlock[nblk] (32 B each), then the packed
 * 32-bit words, with two zero words of padding after the last block's bits.
 */
#ifndef PF_CODEC_H
#define PF_CODEC_H

#include <stdint.h>

#ifdef __CUDACC__
#define PFC_HD __host__ __device__ __forceinline__
#else
#define PFC_HD static inline
#endif

#define PFC_MAGIC 0x31434650u /* "PFC1" */
#define PFC_BLOCK 1024
#define PFC_RAW 0
#define PFC_FOR 1
#define PFC_DELTA 2
#define PFC_RLE 3
/* RLE pages keep at most this many runs (a decoder stages them on chip). */
#define PFC_RLE_MAX_RUNS 4096

typedef struct {
  uint32_t magic;
  uint8_t scheme;
  uint8_t esize;
  uint16_t reserved;
  uint32_t n;      /* rows */
  uint32_t nruns;  /* RLE: runs */
  uint32_t s0;     /* byte offset of stream 0 */
  uint32_t s1;     /* byte offset of stream 1 (RLE) */
  uint32_t bytes;  /* page bytes */
  uint32_t pad[9];
} PfcPage;

typedef struct {
  uint32_t scheme; /* PFC_FOR or PFC_DELTA */
  uint32_t n;
  uint32_t nblk;
  uint32_t pad;
} PfcStream;

typedef struct {
  int64_t base;      /* minimum of the block's (delta) values */
  int64_t first;     /* DELTA: the block's first value */
  uint32_t word_off; /* first 32-bit word of the block's bits, after the block table */
  uint32_t bw;       /* bits per value, 0..64 */
  uint32_t pad[2];
} PfcBlock;

/* The bw-bit field number j of a bitstream starting at words. */
PFC_HD uint64_t pfc_bits(const uint32_t* words, uint32_t j, uint32_t bw) {
  if (bw == 0) return 0;
  const uint64_t bit = (uint64_t)j * bw;
  const uint32_t w = (uint32_t)(bit >> 5), sh = (uint32_t)(bit & 31);
  const uint64_t a = (uint64_t)words[w] | ((uint64_t)words[w + 1] << 32);
  uint64_t v = a >> sh;
  if (sh + bw > 64) v |= (uint64_t)words[w + 2] << (64 - sh);
  if (bw < 64) v &= ((uint64_t)1 << bw) - 1;
  return v;
}

PFC_HD const PfcStream* pfc_stream(const uint8_t* page, uint32_t off) {
  return (const PfcStream*)(page + off);
}
PFC_HD const PfcBlock* pfc_blocks(const PfcStream* s) { return (const PfcBlock*)(s + 1); }
PFC_HD const uint32_t* pfc_words(const PfcStream* s) {
  return (const uint32_t*)(pfc_blocks(s) + s->nblk);
}

/* FOR: value j of a stream.  DELTA needs a scan: pfc_delta_term gives the
 * term that a block's inclusive scan from `first` adds at position j. */
PFC_HD int64_t pfc_for_value(const PfcStream* s, uint32_t j) {
  const PfcBlock* b = pfc_blocks(s) + (j / PFC_BLOCK);
  return (int64_t)((uint64_t)b->base + pfc_bits(pfc_words(s) + b->word_off, j % PFC_BLOCK, b->bw));
}
PFC_HD int64_t pfc_delta_term(const PfcStream* s, uint32_t j) {
  const PfcBlock* b = pfc_blocks(s) + (j / PFC_BLOCK);
  if (j % PFC_BLOCK == 0) return b->first;
  return (int64_t)((uint64_t)b->base + pfc_bits(pfc_words(s) + b->word_off, j % PFC_BLOCK, b->bw));
}

#endif /* PF_CODEC_H */
