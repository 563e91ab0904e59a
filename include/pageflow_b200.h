/*
 * pageflow_b200 — the C ABI of the B200 (sm_100a) relational hot path.
 *
 * Every entry point takes plain device pointers, element counts and a
 * cudaStream_t (passed as void*), returns an int status (PF_OK or a negative
 * PF_E* code; pf_last_error() gives the message of the calling thread's last
 * failure) and allocates no device memory: scratch comes from a caller-owned
 * device workspace whose size the matching *_workspace() function reports,
 * starting on a 256-byte boundary (cudaMalloc's and torch's allocations do;
 * a workspace that does not is refused with PF_ENOSPACE).
 * Outputs are caller-allocated device buffers sized as each function states.
 * A "host_out" argument is caller-owned PINNED host memory (cudaHostAlloc or
 * cudaHostRegister) that a kernel writes through its device alias.
 *
 * Functions that return a row count to the host wait for it once (a bounded
 * poll of one CUDA event; PF_ETIMEOUT after pf_set_wait_timeout_ms()); all
 * other work stays queued on the stream.
 *
 * Reference interfaces replaced (PageFlow, operators/kernels/tqpkernels.cu:8-46,
 * the pybind module TQPlib.tqpkernels):
 *   pf_partition_sort      <- partition_sort     (operators/kernels/partition_sort.cu:610-768)
 *   pf_join_unique_hash    <- join_unique_hash   (operators/kernels/join_core.cu:301-351)
 *   pf_join_semi_anti      <- join_semi_anti     (operators/kernels/join_core.cu:358-400)
 *   pf_join_expand_prepare
 *   + pf_join_expand       <- join_expand        (operators/kernels/join_core.cu:263-295)
 * and the torch tensor programs of the aggregation path:
 *   pf_slab_add / pf_slab_finish <- DenseAggregationSlab.add/finish (operators/aggregation_slab.py:213-246)
 *   pf_join_aggregate      <- the partition -> unique-hash join -> index_select ->
 *                             KeyedAggregate.pass1 -> reduce_tick_slice composition
 *                             (uvm/join.py:98-225, uvm/aggregate.py:147-212)
 */
#ifndef PAGEFLOW_B200_H
#define PAGEFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------ */
#define PF_OK 0
#define PF_EINVAL (-1)   /* an argument outside the function's limits        */
#define PF_ECUDA (-2)    /* a CUDA runtime call failed                        */
#define PF_ETIMEOUT (-3) /* a bounded host or device wait gave up             */
#define PF_ENOSPACE (-4) /* the workspace is smaller than *_workspace() asked */
#define PF_EDEVICE (-5)  /* a kernel raised its device error word             */

/* The calling thread's last failure message ("" after a success). */
const char* pf_last_error(void);
/* Library version, e.g. "0.1.0". */
const char* pf_version(void);
/* The bound of every host wait, in milliseconds (default 120000). */
void pf_set_wait_timeout_ms(int64_t ms);
/* Kernels this library has launched in the process so far. */
int64_t pf_launch_count(void);
/*
 * Per-kernel timing of the calling thread's launches: between
 * pf_profile_begin() and pf_profile_end() every launch is bracketed by a pair
 * of CUDA events on its stream.  pf_profile_end waits for them and fills, for
 * up to max_kernels distinct kernels, its name (name_len bytes a slot), the
 * summed milliseconds and the launches; returns the number of distinct
 * kernels (or a negative PF_E* code).  No counterpart in the reference: it
 * serves the benchmark's live roofline figures.
 */
void pf_profile_begin(void);
int pf_profile_end(int max_kernels, char* names, int name_len, double* total_ms,
                   int64_t* launches);

/* ---- limits (kept equal to the reference's) ----------------------------- */
#define PF_PART_MAX_COLS 6     /* partition_sort.cu:54 MAXC                 */
#define PF_PART_MAX_WIDTHS 4   /* partition_sort.cu:55 MAXCLS (gidx incl.)  */
#define PF_PART_B_MAX 512      /* partition_sort.cu:56 BMAX == JOIN_B_MAX   */
#define PF_JOIN_MAX_ROWS ((int64_t)2147418112) /* join_core.cu:49, 2^31-2^16 */

/* ---- radix partition (drop-in for tqpkernels.partition_sort) ------------ */
/*
 * Stable hash partition of up to 6 columns plus the int64 global index into
 * B padded buckets.  A row's bucket is the top log2(B) bits of mix64(key)
 * (0 when B == 1); rows keep their domain order inside a bucket; each
 * non-empty bucket starts on a whole lcm(row_bytes, 512)-byte unit of its
 * output (rows_per_unit = 512 / gcd(row_bytes, 512)); padding rows are left
 * unwritten.
 *
 *  cols_in[c]    column c: n_dom rows (raw) or n_valid rows (comp[c] = 1,
 *                already compacted by the mask), row_bytes[c] bytes a row
 *  cols_out[c]   n_valid + B*(rows_per_unit(row_bytes[c]) - 1) rows
 *  key_idx       the int64 key column
 *  mask          NULL, or n_dom bytes (non-zero = kept)
 *  n_dom         the mask's rows (or the key's rows without a mask), < 2^31
 *  n_valid       the kept rows (the rows of a compacted column)
 *  goff          global index of domain row 0; gidx = goff + pre-mask row
 *  B             power of two in [1, 512]
 *  select_first  with a mask: collect the kept rows' ids first
 *  gidx_out      int64, n_valid + B*(rows_per_unit(8) - 1) rows
 *  host_out      pinned int64[B + 5]: [0,B) bucket counts; [B, B+4) each
 *                row-width class's padded total (classes numbered by first
 *                appearance over the columns, then the gidx's 8 B); [B+4] the
 *                kept rows a mask prologue found, or -1 when none ran.
 * A kept-row count that the mask contradicts leaves the outputs unwritten
 * (nothing is read or written past what n_valid sizes); the caller compares
 * host_out against n_valid.  Waits once, for the counts.
 */
size_t pf_partition_sort_workspace(int64_t n_dom, int64_t n_valid, int B, int has_mask,
                                   int select_first);
int pf_partition_sort(const void* const* cols_in, void* const* cols_out, const int* row_bytes,
                      const int* comp, int ncols, int key_idx, const uint8_t* mask, int64_t n_dom,
                      int64_t n_valid, int64_t goff, int B, int select_first, int64_t* gidx_out,
                      int64_t* host_out, void* workspace, size_t workspace_bytes, void* stream);
/* 512 / gcd(row_bytes, 512): rows of one padding unit. */
int64_t pf_rows_per_unit(int64_t row_bytes);

/* ---- join cores (drop-ins for join_unique_hash / join_semi_anti / join_expand) */
/*
 * Inner join on a unique build tuple of 1 or 2 int64 keys.  build_idx and
 * probe_idx have n_probe rows each; the first host_out[0] hold the matches in
 * probe-row order.  host_out: pinned int64[2] ([1] is set to 0).  Waits once.
 * 1 <= n_build, n_probe <= PF_JOIN_MAX_ROWS.
 */
size_t pf_join_unique_hash_workspace(int64_t n_build, int64_t n_probe);
int pf_join_unique_hash(const int64_t* build0, const int64_t* build1, int64_t n_build,
                        const int64_t* probe0, const int64_t* probe1, int64_t n_probe, int nkeys,
                        int64_t* build_idx, int64_t* probe_idx, int64_t* host_out,
                        void* workspace, size_t workspace_bytes, void* stream);
/*
 * No counterpart in the reference.  pf_join_unique_hash for callers that may
 * not allocate: no workspace argument and no device allocation by the
 * library; its scratch is one fixed device array of
 * PF_UH_STATIC_SCRATCH_BYTES (8 MiB + 64 KiB) inside the library.  A call
 * fits when 8 * n_build + 4 * n_probe bytes, plus 8 bytes per 4096 probe
 * rows of block counts, stay within it: 524288 build rows with 1048576
 * probe rows is one such call, and so is 1000000 build rows with 10 probe
 * rows.  Larger calls return PF_EINVAL before anything is queued.  The match
 * count goes to match_count (device int64[1]) on the stream; nothing waits.
 * The first call on a device, with that device current, sets the scratch up
 * (looks up its device address, loading the library's module there); make
 * it before any stream capture.  Every call takes the device that is
 * current when it is made, so `stream` must belong to that device.  The
 * address is kept for the life of the process: after cudaDeviceReset it
 * names memory of the destroyed context, so do not call this entry point on
 * a device after resetting it.  The scratch is shared per device: calls
 * that overlap on one device (two streams, two host threads) race.
 */
#define PF_UH_STATIC_SCRATCH_BYTES ((8u << 20) + (64u << 10))
int pf_join_unique_hash_static(const int64_t* build0, const int64_t* build1, int64_t n_build,
                               const int64_t* probe0, const int64_t* probe1, int64_t n_probe,
                               int nkeys, int64_t* build_idx, int64_t* probe_idx,
                               int64_t* match_count, void* stream);

/*
 * Late materialization: rows idx[0, n) of ncols columns (up to 16) in one
 * launch, replacing the per-column torch.index_select / index_with_null of
 * the reference's join tail (operators/hashjoin.py:355-377,
 * conversion.py:39-50).  Column c has row_bytes[c]-byte rows of
 * elem_bytes[c]-byte elements (1, 2, 4, 8) and n_src rows.  With allow_null,
 * an index equal to null_idx gives a row of null_elem[c] elements (the bit
 * pattern of the column's null value, e.g. -64 as that dtype); an index
 * outside [0, n_src) gives that row too and is counted in bad[0] (device
 * int64, added to).  Queued only.
 */
int pf_gather(const void* const* cols_in, void* const* cols_out, const int* row_bytes,
              const int* elem_bytes, const uint64_t* null_elem, int ncols, const int64_t* idx,
              int64_t n, int64_t n_src, int allow_null, int64_t null_idx, int64_t* bad,
              void* stream);

/*
 * Late materialization with zero copy: the same gather from columns held in
 * pinned host memory as segments, read in place over the host link (the
 * reference's zero_copy_rearrange_kernel, IO/zero_copy_reader.cu:89-118, with
 * an error count where it traps).  Segment s of every column holds rows
 * [seg_rows[s], seg_rows[s + 1]) (host int64, ascending, nseg + 1 of them,
 * nseg <= 1024); seg_ptrs[c * nseg + s] is column c's segment s (pinned host
 * memory, cudaHostAlloc or registered).  Output row i of column c is row
 * idx[i] + base; an index equal to null_idx (with allow_null) gives a row of
 * null_elem[c] elements, an index outside the segments that row too, counted
 * in bad[0] (device int64, added to) and never read.  With order (device
 * int64[n], a permutation of [0, n), e.g. the argsort of idx), output rows
 * are taken in that order, so neighbouring threads read neighbouring host
 * rows.  Workspace: pf_gather_segments_workspace(ncols, nseg).  Queued only.
 */
size_t pf_gather_segments_workspace(int ncols, int nseg);
int pf_gather_segments(void* const* seg_ptrs, const int64_t* seg_rows, int nseg, int64_t base,
                       int ncols, const int* row_bytes, const int* elem_bytes,
                       const uint64_t* null_elem, const int64_t* idx, const int64_t* order,
                       int64_t n, int allow_null, int64_t null_idx, void* const* cols_out,
                       int64_t* bad, void* workspace, size_t workspace_bytes, void* stream);

/* Residual operators of a semi/anti summary, as build.v OP probe.v. */
#define PF_OP_NONE 0
#define PF_OP_NE 1
#define PF_OP_LT 2
#define PF_OP_LE 3
#define PF_OP_GT 4
#define PF_OP_GE 5
/*
 * Semi (anti = 0) or anti (anti = 1) join on a hash set of build keys; with
 * op != PF_OP_NONE a match must also pass build_val OP probe_val for some
 * build row of the key (answered by the key's min and/or max).  out has
 * n_probe rows; the first host_out[0] are the kept probe rows, ascending.
 * host_out[1] = 1 when a build key equals INT64_MIN (the empty-slot value;
 * the result is then not valid).  Waits once.
 */
size_t pf_join_semi_anti_workspace(int64_t n_build, int64_t n_probe, int op);
int pf_join_semi_anti(const int64_t* build_key, int64_t n_build, const int64_t* probe_key,
                      int64_t n_probe, const int64_t* build_val, const int64_t* probe_val, int op,
                      int anti, int64_t* out, int64_t* host_out, void* workspace,
                      size_t workspace_bytes, void* stream);

/*
 * Sort/search pair expansion in two calls sharing one workspace:
 * prepare scans len[0,m) and waits for the pair count (host_out[0]); run
 * writes, for every probe row i and j < len[i], the pair
 * (sorted_ids[start[i] + j], i) in probe-row order into cs / cr
 * (host_out[0] rows each).
 */
size_t pf_join_expand_workspace(int64_t m);
int pf_join_expand_prepare(const int64_t* len, int64_t m, int64_t* host_out, void* workspace,
                           size_t workspace_bytes, void* stream);
int pf_join_expand(const int64_t* sorted_ids, const int64_t* start, const int64_t* len, int64_t m,
                   int64_t n_pairs, int64_t* cs, int64_t* cr, void* workspace,
                   size_t workspace_bytes, void* stream);

/* ---- dense slab group-by (DenseAggregationSlab) -------------------------- */
#define PF_AGG_SUM 0
#define PF_AGG_MAX 1
#define PF_AGG_MIN 2
#define PF_DT_I64 0
#define PF_DT_F64 1
#define PF_DT_I32 2
/*
 * Fold n rows into a direct-addressed slab over [key_min, key_min + capacity):
 * occupied[key - key_min] = 1 and values[v][(key - key_min) * width[v] + e]
 * op= src[v][row * width[v] + e].  keys are int64 (key_dtype PF_DT_I64) or
 * int32 (PF_DT_I32); every key must lie in the range (rows outside it are
 * counted into err_count, a device int64, and skipped).  Queued only.
 */
int pf_slab_add(const void* keys, int key_dtype, int64_t n, int64_t key_min, int64_t capacity,
                uint8_t* occupied, int nvals, void* const* values, const void* const* srcs,
                const int* dtypes, const int* ops, const int* widths, int64_t* err_count,
                void* stream);
/*
 * The occupied slots, ascending: keys_out[j] = key_min + slot and
 * vals_out[v][j] = values[v][slot] for the first host_out[0] rows (outputs
 * sized for `capacity` rows).  Waits once.
 */
size_t pf_slab_finish_workspace(int64_t capacity);
int pf_slab_finish(const uint8_t* occupied, int64_t key_min, int64_t capacity, int nvals,
                   const void* const* values, const int* dtypes, const int* widths,
                   int64_t* keys_out, void* const* vals_out, int64_t* host_out, void* workspace,
                   size_t workspace_bytes, void* stream);

/* ---- fused radix partition -> build/probe -> slab group-by --------------- */
/*
 * SELECT group, SUM(price * (scale - disc)), COUNT(*) FROM build JOIN probe
 * ON build.key = probe.fk GROUP BY build.group, with a unique build key.
 * Both sides are partitioned by the top log2(B) bits of mix64(key)
 * (B a power of two in [1, 4096]), each partition's build rows go into an
 * open-addressing table, and each matched probe row adds its value into a
 * dense slab over [group_min, group_min + n_groups).  probe_disc may be NULL
 * (the value is then price).  Sums are exact int64 (wrapping on overflow as
 * int64 arithmetic does).  Outputs: sum_out / count_out [n_groups] (zero for
 * groups no row reached; a group is present iff its count > 0) and, in
 * stats_out (device int64[4]): matched probe rows, the device error word (0,
 * or nonzero when a kernel gave up a bounded wait for its bulk copies; the
 * outputs are then not valid), build rows whose group is out of range (their
 * matches are not aggregated), and the number of build rows no table slot
 * took (0 on success).
 *
 * The default (shared-memory) path counts no rows before it scatters: each
 * bucket of the first radix pass, and each sub-bucket of the second, owns a
 * region sized for its expected rows plus seven standard deviations (eight
 * times the mean's variance on the probe side, whose keys repeat), and a
 * pass whose region would overflow (skewed keys) is run again after counting
 * its rows exactly.  The second pass is planned on the device from the first
 * pass's cursors, so the call waits once, at the end, for both passes'
 * overflow words (and again only when one overflowed); with
 * PF_JOIN_PATH=rounds it waits once, for the bucket counts that plan the
 * rounds, and the rest stays queued.
 */
size_t pf_join_aggregate_workspace(int64_t n_build, int64_t n_probe, int B, int64_t n_groups);
int pf_join_aggregate(const int64_t* build_key, const int32_t* build_group, int64_t n_build,
                      const int64_t* probe_fk, const int64_t* probe_price,
                      const int64_t* probe_disc, int64_t scale, int64_t n_probe, int B,
                      int64_t group_min, int64_t n_groups, int64_t* sum_out, int64_t* count_out,
                      int64_t* stats_out, void* workspace, size_t workspace_bytes, void* stream);
/*
 * The run-time choices of a fused join + group-by, the autotuner's knobs
 * beside the fan-out B (pageflow_b200/autotune.py times candidates on a
 * shape's first call and caches the fastest).  No counterpart in the
 * reference, whose fan-out comes from its partition-count rule alone
 * (operators/partitions.py:54-85).
 *   path      0: the shared-memory join (second radix pass, a table per
 *             sub-partition in shared memory); 1: L2 rounds (one radix pass,
 *             tables in L2; a smaller workspace)
 *   table     shared-memory join: 0 a table of 8-byte hash slots, 1 4-byte
 *             fingerprinted slots with the build hashes and cells by row
 *   sub_rows  build rows a sub-partition aims at (0: 1365); fewer rows, more
 *             sub-partitions in the second radix pass
 *   counted   1: both radix passes count their rows before they scatter
 *             (else only a pass whose regions overflowed)
 * With knobs = NULL the defaults apply (overridden, for sweeps, by
 * PF_JOIN_PATH=rounds|smem, PF_SJ_FP, PF_SJ_TARGET and PF_COUNTED).  The
 * workspace depends on the knobs: query it with the same ones.
 */
typedef struct pf_join_knobs {
  int path;
  int table;
  int sub_rows;
  int counted;
} pf_join_knobs;
size_t pf_join_aggregate_workspace_ex(int64_t n_build, int64_t n_probe, int B, int64_t n_groups,
                                      const pf_join_knobs* knobs);
int pf_join_aggregate_ex(const int64_t* build_key, const int32_t* build_group, int64_t n_build,
                         const int64_t* probe_fk, const int64_t* probe_price,
                         const int64_t* probe_disc, int64_t scale, int64_t n_probe, int B,
                         int64_t group_min, int64_t n_groups, int64_t* sum_out,
                         int64_t* count_out, int64_t* stats_out, const pf_join_knobs* knobs,
                         void* workspace, size_t workspace_bytes, void* stream);
/*
 * The fused join + group-by sharded over ranks, in its two rank-local
 * phases (no counterpart in the reference, which runs on one GPU; the
 * exchange between them is the caller's, e.g. NCCL all-to-alls):
 *
 * pf_join_partition: a rank's rows hashed and radix-partitioned into B
 * buckets (B a power of two <= 4096; bucket = top log2(B) bits of
 * mix64(key)), counted first so that every bucket is contiguous, in bucket
 * order: build rows as build_hash_out[n_build] (mix64 of the key) and
 * build_group_out[n_build], probe rows as probe_rec_out[2 * n_probe]
 * records {mix64(fk), price * (scale - disc)} (price when disc is NULL).
 * host_counts (host int64[2B]): each bucket's build rows, then its probe
 * rows.  Waits once, for the counts.
 *
 * pf_join_aggregate_buckets: the second radix pass and the join over nbk
 * buckets a rank holds, each bucket's rows contiguous and the buckets one
 * after another on each side (counts: host int64[2 * nbk], build rows of
 * every bucket, then probe rows; every row of a bucket shares the top logB
 * bits of its hash), into sum_out / count_out [n_groups] over [group_min,
 * group_min + n_groups) and stats_out as pf_join_aggregate's.  Knobs as
 * pf_join_aggregate_ex's (the shared-memory join only).  Adding the ranks'
 * slabs gives the join's result.  Waits at the end unless both sides'
 * second pass was counted.
 */
size_t pf_join_partition_workspace(int64_t n_build, int64_t n_probe, int B);
int pf_join_partition(const int64_t* build_key, const int32_t* build_group, int64_t n_build,
                      const int64_t* probe_fk, const int64_t* probe_price,
                      const int64_t* probe_disc, int64_t scale, int64_t n_probe, int B,
                      int64_t* build_hash_out, int32_t* build_group_out, int64_t* probe_rec_out,
                      int64_t* host_counts, void* workspace, size_t workspace_bytes,
                      void* stream);
size_t pf_join_aggregate_buckets_workspace(const int64_t* counts, int nbk, int64_t n_groups,
                                           const pf_join_knobs* knobs);
int pf_join_aggregate_buckets(const int64_t* build_hash, const int32_t* build_group,
                              const int64_t* probe_rec, const int64_t* counts, int nbk,
                              int logB, int64_t group_min, int64_t n_groups, int64_t* sum_out,
                              int64_t* count_out, int64_t* stats_out,
                              const pf_join_knobs* knobs, void* workspace,
                              size_t workspace_bytes, void* stream);
/* The fan-out the autotuner seeds pf_join_aggregate with for these sizes. */
int pf_join_aggregate_pick_b(int64_t n_build, int64_t n_probe);
/*
 * Which passes the calling thread's last pf_join_aggregate counted before it
 * scattered: bit 0 the first radix pass, bit 1 the second (both taken again
 * after a region overflowed, or forced with PF_COUNTED=1).  No counterpart in
 * the reference, whose partition kernel always counts first.
 */
int pf_join_aggregate_counted_passes(void);
/*
 * The groups a dense (sum, count) slab holds, ascending: keys_out[j] =
 * group_min + g, sums_out[j] = sum[g], counts_out[j] = count[g] for every g
 * with count[g] > 0; host_out[0] = their number (outputs sized n_groups).
 * The finish of DenseAggregationSlab (operators/aggregation_slab.py:241-246)
 * with COUNT as the occupancy.  Waits once.
 */
size_t pf_groups_finish_workspace(int64_t n_groups);
int pf_groups_finish(const int64_t* sum, const int64_t* count, int64_t group_min,
                     int64_t n_groups, int64_t* keys_out, int64_t* sums_out, int64_t* counts_out,
                     int64_t* host_out, void* workspace, size_t workspace_bytes, void* stream);

/* ---- hash route of the keyed aggregation (pass 1) --------------------------- */
/*
 * Each row's grouping hash (KeyedAggregate.pass1's linear hash,
 * operators/aggregate.py:551-564): key column c has row_bytes[c]-byte rows,
 * read as little-endian int64 words zero-padded to a multiple of 8 bytes
 * (_pack_as_int64, :482-505); hash = sum over columns and words of word *
 * coeffs[c][word], int64 wrap-around.  coeffs[c]: device int64[ceil(
 * row_bytes[c] / 8)].  Up to 8 key columns.  Queued only.
 */
int pf_group_hash(const void* const* key_cols, const int* row_bytes, const int64_t* const* coeffs,
                  int ncols, int64_t n, int64_t* hash_out, void* stream);
/*
 * Each hash's bucket among B (a power of two <= 4096): the top log2(B) bits
 * of its mix64 (_bucket_ids, operators/aggregate.py:107-116), int32; and
 * the rows per bucket into counts_out (device int64[B], overwritten).
 */
int pf_hash_buckets(const int64_t* hash, int64_t n, int B, int32_t* bucket_out,
                    int64_t* counts_out, void* stream);

/* ---- sorted runs of the two-pass aggregation -------------------------------- */
/*
 * Stable ascending sort of n int64 keys carrying int64 values (vals_in NULL:
 * the row numbers): LSD radix sort over the key range; waits once (for the
 * range).  Outputs n rows each.
 */
size_t pf_sort_pairs_workspace(int64_t n);
int pf_sort_pairs(const int64_t* keys_in, const int64_t* vals_in, int64_t n, int64_t* keys_out,
                  int64_t* vals_out, void* workspace, size_t workspace_bytes, void* stream);
/*
 * Value columns of the run primitives: kinds[q] 0 = integer, 1 = float;
 * esizes[q] 4 or 8; widths[q] elements a row (a (rows, width) tensor);
 * ops[q] 0 = sum, 1 = amax, 2 = amin (operators/sorted_run_merge.py
 * MERGEABLE_OPS).  Up to 16 columns.
 *
 * reduce_tick_slice (operators/sorted_run_merge.py:62-92): the unique keys
 * of keys[0, n) ascending into keys_out and, per value column, each key's
 * rows reduced by its op (the first row starts the reduction, as
 * include_self=False does) into vals_out[q] (n_unique rows).  *n_unique
 * (host) gets the unique count; waits twice.  Integer sums wrap as int64;
 * float sums are added in no fixed order.
 */
size_t pf_unique_reduce_workspace(int64_t n);
int pf_unique_reduce(const int64_t* keys, int64_t n, int ncols, const void* const* vals_in,
                     void* const* vals_out, const int* kinds, const int* esizes,
                     const int* widths, const int* ops, int64_t* keys_out, int64_t* n_unique,
                     void* workspace, size_t workspace_bytes, void* stream);
/*
 * merge_sorted_unique_runs_inplace (operators/sorted_run_merge.py:94-174),
 * out of place: the union of the ascending unique runs run_keys[0, n_run)
 * and tick_keys[0, n_tick) into out_keys (n_run + n_tick rows of room), a
 * key in both taking op(run value, tick value); *n_out (host) gets the
 * merged length; waits once.
 */
size_t pf_merge_sorted_runs_workspace(int64_t n_tick);
int pf_merge_sorted_runs(const int64_t* run_keys, const void* const* run_vals, int64_t n_run,
                         const int64_t* tick_keys, const void* const* tick_vals, int64_t n_tick,
                         int ncols, const int* kinds, const int* esizes, const int* widths,
                         const int* ops, int64_t* out_keys, void* const* out_vals, int64_t* n_out,
                         void* workspace, size_t workspace_bytes, void* stream);

/* ---- compressed pages: decode on arrival, filter, partition ---------------- */
/*
 * PFC1 pages (pageflow_b200/csrc/codec.h): a page holds up to 2^30 values of
 * one int32/int64 column, encoded with the smallest of FOR bitpacking, DELTA
 * + FOR, RLE (run values FOR or DELTA, run ends DELTA) or RAW, in
 * independently decodable 1024-value mini-blocks.  Replaces the reference's
 * nvCOMP CASCADED codec (compression/nvcomp_manager.cu:162-173) with a format
 * of our own.  pf_page_encode (host) writes one page into out; returns its
 * bytes or a negative PF_E* code.
 */
int64_t pf_page_encode(const void* values, int esize, int64_t n, void* out, int64_t capacity);
/*
 * Output-side encoding on the device: an int32/int64 column (values, device,
 * esize 4 or 8) cut into npages pages, page p = rows [page_rows[p],
 * page_rows[p + 1]) (host int64, at most 2^30 rows a page; e.g. the buckets
 * of a partitioned output), each written as a PFC1 page into out (device,
 * capacity bytes), byte for byte the page pf_page_encode writes for the same
 * values.  page_offsets (host int64[npages + 1]) receives each page's byte
 * offset and the total.  The device counterpart of the reference's
 * compression of partitioned outputs (IO/codec/region_producer.py, layout
 * IO/codec/batched_compress.py:27-59), with this library's format.  Waits
 * once, for the page sizes; PF_ENOSPACE when the pages exceed capacity
 * (nothing written).
 */
size_t pf_encode_pages_workspace(int npages);
int pf_encode_pages(const void* values, int esize, const int64_t* page_rows, int npages,
                    void* out, int64_t capacity, int64_t* page_offsets, void* workspace,
                    size_t workspace_bytes, void* stream);
/*
 * The paged benchmark's probe table generated and encoded on host threads:
 * n_rows rows of 6 columns (fk int64 with Zipf ranks from the given table over
 * n_build keys, date int32 sorted within 2^20-row runs in [8035, 10591],
 * price int64, quantity int64, flag int32, status int32), rows_per_page rows
 * a row group.  pf_paged_fetch copies the pages (group-major, columns in
 * order) into dst and each page's byte offset into directory[n_groups * 6],
 * and frees the handle.
 */
int pf_paged_generate(uint64_t seed, int64_t n_rows, int rows_per_page, int64_t n_build,
                      const int64_t* zipf_edges, const uint64_t* zipf_thr, int nbins, int threads,
                      void** handle, int64_t* total_bytes);
int pf_paged_fetch(void* handle, void* dst, int64_t* directory, int64_t* n_groups);
/*
 * Decode on arrival: batches of groups_per_batch row groups are copied from
 * pinned host pages (host_pages, total_bytes; directory as pf_paged_fetch
 * writes it, host memory) to the device on a copy stream, NSTAGE batches
 * ahead, while `stream` decodes each batch, keeps the rows with lo <=
 * column[filter_col] < hi, and scatters their other columns into outs[c]
 * (device, capacity_rows rows each; NULL to drop a column) by the key
 * column's radix bucket (top log2(B) bits of mix64).  Each batch's rows form
 * one region of the outputs, bucket after bucket: bucket_offsets (device,
 * [n_batches][B + 1]) receives each bucket's first output row (-1 when the
 * batch did not fit the capacity and was skipped) and the batch's rows.
 * stats (device int64[4]): rows written, batches skipped, bad pages.  Queued
 * only.  The pages are trusted input (written by pf_page_encode /
 * pf_paged_generate).
 */
size_t pf_paged_scan_workspace(const int64_t* directory, int64_t n_groups, int ncols,
                               int64_t total_bytes, int groups_per_batch, int B);
int pf_paged_scan(const uint8_t* host_pages, const int64_t* directory, int64_t n_groups, int ncols,
                  const int* esizes, int64_t total_bytes, int64_t n_rows, int rows_per_page,
                  int filter_col, int64_t lo, int64_t hi, int key_col, int B,
                  int groups_per_batch, void* const* outs, int64_t capacity_rows,
                  int64_t* bucket_offsets, int64_t* stats, void* workspace,
                  size_t workspace_bytes, void* stream);

/* ---- batched join -> group-by (many uneven instances, one launch) --------- */
/*
 * One instance: SELECT group, SUM(value), COUNT(*) FROM build JOIN probe ON
 * build.key = probe.fk GROUP BY build.group, a unique build key, groups in
 * [group_min, group_min + n_groups).  Device pointers; 0 rows allowed.
 */
typedef struct {
  const int64_t* build_key;
  const int32_t* build_group;
  int64_t n_build;
  const int64_t* probe_fk;
  const int64_t* probe_value;
  int64_t n_probe;
  int64_t group_min;
  int64_t n_groups;
} pf_batch_instance;
/*
 * The batch engine: pf_batch_prepare uploads the instances' descriptors into
 * the workspace and lays out a hash table per instance (twice its build rows
 * in 16-byte slots) and a dense (sum, count) slab per instance; it waits
 * once.  pf_batch_run then queues only device work (a reset of the slabs and
 * the work counters, then one persistent launch in which blocks take build
 * and probe work items from a device queue, a probe item waiting, bounded,
 * for its instance's build items), so it can be captured in a CUDA graph and
 * replayed; each run bumps a device epoch that tags the table slots, so the
 * tables are never cleared.  pf_batch_slab gives instance i's slab: int64
 * pairs (sum, count) per group, interleaved.  stats (device int64[4]):
 * matched probe rows, device error word (a bounded wait gave up), build rows
 * out of group range, table overflows.  No counterpart in the reference
 * (which launches per instance); it serves the batching workload.
 */
size_t pf_batch_workspace(const pf_batch_instance* instances, int n);
int pf_batch_prepare(const pf_batch_instance* instances, int n, void* workspace,
                     size_t workspace_bytes, void* stream);
int pf_batch_run(void* workspace, int64_t* stats, void* stream);
int64_t* pf_batch_slab(void* workspace, int i);

/* ---- serving: resident dimension tables, requests in persistent launches -- */
/*
 * A dimension table's hash table, built once and kept across requests:
 * 16-byte slots, a power of two of at least 2 x n_keys.  Keys must be unique
 * (as the reference's unique-hash join requires of its build side); groups
 * outside [0, n_groups) are kept but never aggregated.  stats (device
 * int64[2]): rows with a group out of range, rows that found no slot.
 */
size_t pf_dim_table_bytes(int64_t n_keys);
int pf_dim_build(const int64_t* keys, const int32_t* groups, int64_t n_keys, int64_t n_groups,
                 void* table, size_t table_bytes, int64_t* stats, void* stream);
/*
 * One request's share of a launch: SELECT group, SUM(value), COUNT(*) FROM
 * probe JOIN dim ON probe.fk = dim.key WHERE date_lo <= probe.date < date_hi
 * GROUP BY dim.group, over the probe rows [row_begin, row_end) of this
 * launch.  slab: device int64[2 x n_groups] (sum, count) pairs, zero before
 * the request's first launch, accumulated across its launches.  In the
 * launch with finish = 1 the occupied groups are written in ascending order
 * (out_keys / out_sums / out_counts, n_groups rows each; out_n the count)
 * and the pinned host word *done (may be NULL) is set to 1 + groups once
 * they are written (all ones if the launch gave up on it).  n_groups <=
 * 4,194,304.
 */
typedef struct {
  const void* table;
  int64_t n_keys;
  int64_t n_groups;
  const int64_t* fk;
  const int32_t* date;
  const int64_t* value;
  int64_t row_begin, row_end;
  int32_t date_lo, date_hi;
  int32_t finish;
  int32_t pad;
  int64_t* slab;
  int64_t* out_keys;
  int64_t* out_sums;
  int64_t* out_counts;
  int64_t* out_n;
  int64_t* done;
} pf_serve_request;
/*
 * One persistent launch over n requests (1 <= n <= 8192), in the order given
 * (a request's items run before the next request's are handed out).  Queued only; the
 * request list is staged through pinned memory of the calling thread.
 * stats (device int64[4], zeroed by the caller, added to by every launch):
 * matched rows, device error word (a bounded wait gave up; the request's
 * done word is then set to all ones), rows that passed the filter.  No counterpart in the reference:
 * it serves the serving workload (requests against resident tables).
 */
size_t pf_serve_workspace(int max_requests);
int pf_serve_run(const pf_serve_request* requests, int n, void* workspace,
                 size_t workspace_bytes, int64_t* stats, void* stream);

/* ---- seeded synthetic inputs (identical to the CPU generator) ------------ */
/* config ids: 0 = small (250K x 1M, 25 groups), 1 = scale (150M x 600M,
 * 1.5M groups); `rows` and `lo` select rows [lo, lo + rows). */
int pf_gen_build(int config, uint64_t seed, int64_t n_build, int64_t n_groups, int64_t lo,
                 int64_t rows, int64_t* key, int32_t* group, void* stream);
int pf_gen_probe(int config, uint64_t seed, int64_t n_build, int64_t lo, int64_t rows,
                 int64_t* fk, int64_t* price, int64_t* disc, void* stream);
/* One batching instance's probe rows: FK ranks drawn from the Zipf table
 * (nbins bins: edges[nbins+1] ranks, thr[nbins] cumulative thresholds, both
 * device arrays), values in cents. */
int pf_gen_batch_probe(uint64_t seed, int64_t n_build, int64_t lo, int64_t rows, int nbins,
                       const int64_t* edges, const uint64_t* thr, int64_t* fk, int64_t* value,
                       void* stream);
/* The serving workload: dimension rows [lo, lo + rows) of a dimension of
 * n_keys keys (the n_keys most referenced of n_ranks ranks), and fact rows
 * (FK ranks from the Zipf table, dates, values). */
int pf_gen_serve_dim(uint64_t seed, int64_t n_ranks, uint64_t group_seed, int64_t n_keys,
                     int64_t n_groups, int64_t lo, int64_t rows, int64_t* key, int32_t* group,
                     void* stream);
int pf_gen_serve_fact(uint64_t seed, int64_t n_ranks, int nbins, const int64_t* edges,
                      const uint64_t* thr, int64_t lo, int64_t rows, int64_t* fk, int32_t* date,
                      int64_t* value, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PAGEFLOW_B200_H */
