/*
 * jfx.h -- C ABI of the B200 (sm_100a) kernels behind jaxframes' distributed
 * algorithms layer (src/jaxframes/distributed/parallel_algorithms.py).
 *
 * Every entry point takes plain device pointers, element counts, a caller-owned
 * device workspace (size from jfx_workspace_size, 256-byte aligned as
 * cudaMalloc returns it; a misaligned one is JFX_ERR_ARG) and a cudaStream_t
 * passed as void*.  Work is stream-ordered; entry points that must size an output (group
 * count, join pair count) synchronise the stream once and return the size
 * through a host pointer, as the reference does with its host reads at
 * parallel_algorithms.py:712, :772 and :880.
 *
 * Return value: JFX_OK (0) or a negative jfx_status; jfx_last_error() gives a
 * thread-local message.  Nothing here falls back to the CPU.
 */
#ifndef JFX_H
#define JFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  JFX_OK = 0,
  JFX_ERR_ARG = -1,      /* bad argument (null pointer, bad count, bad flag) */
  JFX_ERR_DTYPE = -2,    /* dtype the reference does not sort / aggregate */
  JFX_ERR_ALLOC = -3,    /* workspace too small */
  JFX_ERR_TIMEOUT = -4,  /* a bounded device-side wait gave up */
  JFX_ERR_CAPACITY = -5, /* output capacity or row limit exceeded */
  JFX_ERR_CUDA = -6      /* CUDA runtime error */
} jfx_status;

typedef enum {
  JFX_I8 = 1, JFX_I16 = 2, JFX_I32 = 3, JFX_I64 = 4,
  JFX_U8 = 5, JFX_U16 = 6, JFX_U32 = 7, JFX_U64 = 8,
  JFX_F32 = 9, JFX_F64 = 10, JFX_BOOL = 11
} jfx_dtype;

/* column flags */
#define JFX_COL_DESC 1u /* descending key of multi_column_lexsort (-x / max-x) */

typedef struct {
  const void* data; /* device pointer, n elements, contiguous */
  int32_t dtype;    /* jfx_dtype */
  uint32_t flags;   /* JFX_COL_* */
} jfx_column;

/* aggregation bits (SortBasedGroupBy._apply_aggregation_vectorized,
 * parallel_algorithms.py:626-660, and _scatter_group_aggregate, :1212-1228) */
#define JFX_AGG_SUM 1u
#define JFX_AGG_MEAN 2u
#define JFX_AGG_COUNT 4u
#define JFX_AGG_MIN 8u
#define JFX_AGG_MAX 16u

typedef struct {
  const void* data; /* device pointer to the value column (original row order) */
  int32_t dtype;    /* jfx_dtype of the values */
  uint32_t aggs;    /* JFX_AGG_* bits requested on this column */
  /* outputs, capacity n each, indexed by group; dtypes follow the reference:
   * sum: value dtype; count: value dtype (single key) or int32 (multi key);
   * mean: mean_dtype; min/max: value dtype */
  void* out_sum;
  void* out_mean;
  void* out_count;
  void* out_min;
  void* out_max;
  int32_t mean_dtype; /* JFX_F32 or JFX_F64 */
  int32_t count_dtype;
} jfx_agg_column;

/* join kinds (ParallelSortMergeJoin.join, parallel_algorithms.py:938-1075) */
#define JFX_JOIN_INNER 0
#define JFX_JOIN_LEFT 1
#define JFX_JOIN_RIGHT 2
#define JFX_JOIN_OUTER 3

/* workspace kinds for jfx_workspace_size */
#define JFX_WS_SORT 1      /* n1 = rows */
#define JFX_WS_GROUPBY 2   /* n1 = rows */
#define JFX_WS_JOIN 3      /* n1 = left rows, n2 = right rows */
#define JFX_WS_PARTITION 4 /* n1 = rows, n2 = partitions */
#define JFX_WS_LEARNED 5   /* n1 = rows (uint64 keys) */
#define JFX_WS_BATCH 6     /* n1 = total rows, n2 = queries */

const char* jfx_last_error(void);
int jfx_version(void);
int jfx_max_rows(void);
size_t jfx_workspace_size(int kind, int64_t n1, int64_t n2);

/* ParallelRadixSort.sort (parallel_algorithms.py:463-581) / parallel_sort
 * (:1079-1114): stable ascending order of `key`; ascending==0 reverses the
 * whole result.  Writes the permutation (int32 row ids) and, if non-null, the
 * sorted keys in the key's dtype. */
int jfx_sort(const jfx_column* key, int64_t n, int ascending, int32_t* perm_out,
             void* sorted_keys_out, void* workspace, size_t workspace_bytes, void* stream);

/* jfx_sort without a workspace, for callers that cannot allocate device
 * memory (inside an allocator or memory-pool callback, in loops that must not
 * take cudaMalloc's device-wide synchronisation, or as a plugin that is
 * handed only its input and output buffers).  No counterpart in the
 * reference.  Same arguments, results and errors as jfx_sort; the scratch is a
 * fixed 16 MiB device array inside the library, so n is limited to
 * JFX_SORT_STATIC_MAX_ROWS (JFX_ERR_CAPACITY beyond it).  Allocates nothing:
 * no cudaMalloc / cudaFree and no pinned host memory.  The first call on a
 * device looks up the array's device address; make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller. */
#define JFX_SORT_STATIC_MAX_ROWS 524288
int jfx_sort_static(const jfx_column* key, int64_t n, int ascending, int32_t* perm_out,
                    void* sorted_keys_out, void* stream);

/* multi_column_lexsort (parallel_algorithms.py:25-66): stable lexicographic
 * argsort of ncols columns (first column most significant), JFX_COL_DESC per
 * column.  One column: ascending ignored, as in the reference. */
int jfx_lexsort(const jfx_column* keys, int ncols, int64_t n, int32_t* perm_out,
                void* workspace, size_t workspace_bytes, void* stream);

/* SortBasedGroupBy.groupby_aggregate (:733-803, multi_key=0) and
 * groupby_aggregate_multi_column (:662-731, multi_key=1).  unique_out[c] gets
 * the unique keys of column c (capacity n, ascending / lexicographic order).
 * *num_groups receives G after one stream synchronisation. */
int jfx_groupby(const jfx_column* keys, int ncols, int64_t n, int multi_key,
                const jfx_agg_column* values, int nvalues, void* const* unique_out,
                int64_t* num_groups, void* workspace, size_t workspace_bytes, void* stream);

/* Opaque state passed from jfx_join_prepare to the other join calls
 * (caller-owned plain memory; it points into the workspace, which must stay
 * untouched until the last call that uses the plan). */
typedef struct {
  uint64_t opaque[160];
} jfx_join_plan;

/* ParallelSortMergeJoin.join (:938-1075) and join_multi_column (:826-936),
 * first half: radix sorts both sides by their ncols key columns under one
 * shared key packing and counts, for every row of the driving side, its
 * equal-key run on the other side.  `how`: JFX_JOIN_INNER / LEFT / RIGHT /
 * OUTER (OUTER = inner pairs plus the counts needed for both sides' unmatched
 * rows).  *num_out receives the row count jfx_join_expand writes (inner pairs
 * for INNER/OUTER, one row per left/right row for LEFT/RIGHT) after one stream
 * synchronisation. */
int jfx_join_prepare(const jfx_column* left_keys, int64_t nl, const jfx_column* right_keys,
                     int64_t nr, int ncols, int how, jfx_join_plan* plan, int64_t* num_out,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Second half: writes num_out rows of (left row id, right row id) -- -1 for a
 * missing side -- and, for each non-null keys_out[c], the key column c of the
 * driving side.  Row order is the reference's sorted merge order: inner pairs
 * by (key, left row, right row); left/right rows in that side's sorted order
 * with the first match of the other side (searchsorted, :1013-1034). */
int jfx_join_expand(const jfx_join_plan* plan, int32_t* left_idx_out, int32_t* right_idx_out,
                    void* const* keys_out, void* stream);

/* A payload column gathered by jfx_join_expand_gather as the rows are
 * written: out[i] = data[row] of the output row's left (side 0) or right
 * (side 1) row, converted to out_dtype; a missing row (-1) gives NaN for a
 * float output and -1 otherwise -- the gathers of ParallelSortMergeJoin.join
 * (:1056-1073), which jfx_gather also implements. */
typedef struct {
  const void* data; /* device pointer, n rows of the side's table, original order */
  int64_t n;
  int32_t dtype;
  int32_t side;     /* 0 = left table, 1 = right table */
  void* out;        /* device pointer, num_out elements of out_dtype */
  int32_t out_dtype;
  int32_t reserved;
} jfx_join_payload;

/* jfx_join_prepare that also takes the payload columns jfx_join_expand_gather
 * will write (their `out` is not used here).  A side whose payloads are all
 * 4- or 8-byte and take at most 4 32-bit words in total carries them through
 * its sort, so the expand reads them in sorted order instead of gathering
 * them by row id (not for outer joins or float keys); that side keeps no row
 * ids, so its index output must then be null.  No counterpart in the
 * reference, where the gathers follow the join (:1056-1073). */
int jfx_join_prepare_payloads(const jfx_column* left_keys, int64_t nl, const jfx_column* right_keys,
                              int64_t nr, int ncols, int how, const jfx_join_payload* payloads,
                              int npayloads, jfx_join_plan* plan, int64_t* num_out, void* workspace,
                              size_t workspace_bytes, void* stream);

/* jfx_join_expand plus up to 8 payload gathers in the same kernel (inner,
 * left and right joins; outer joins use jfx_join_expand + jfx_gather).
 * left_idx_out / right_idx_out may be null here. */
int jfx_join_expand_gather(const jfx_join_plan* plan, int32_t* left_idx_out, int32_t* right_idx_out,
                           void* const* keys_out, const jfx_join_payload* payloads, int npayloads,
                           void* stream);

/* Rows of one side (0 = left, 1 = right) that have no match, in ascending row
 * order, as join_multi_column appends them (:883-917).  *count receives the
 * number after one stream synchronisation; rows_out needs that capacity. */
int jfx_join_unmatched(const jfx_join_plan* plan, int side, int32_t* rows_out, int64_t capacity,
                       int64_t* count, void* stream);

/* _coalesce_join_key (:1245-1251): out[i] = left[left_idx[i]] when
 * left_idx[i] >= 0, else right[right_idx[i]] (both columns of `dtype`). */
int jfx_coalesce(const void* left, const int32_t* left_idx, int64_t nl, const void* right,
                 const int32_t* right_idx, int64_t nr, int64_t n, int32_t dtype, void* out,
                 void* stream);

/* Payload gather with the reference's join fill (:1056-1073): out[i] =
 * src[idx[i]] converted to out_dtype, NaN where idx[i] < 0 (float outputs). */
int jfx_gather(const void* src, int32_t src_dtype, int64_t n_src, const int32_t* idx,
               int64_t n, void* out, int32_t out_dtype, void* stream);

/* hash_multi_columns (parallel_algorithms.py:69-136): uint32 per row. */
int jfx_hash_columns(const jfx_column* keys, int ncols, int64_t n, uint32_t* hash_out,
                     void* stream);

/* One device's body of collective_hash_repartition (:163-182, :213-214) with
 * the device count set to num_partitions: target = hash % P and a stable
 * counting sort by target.  Writes targets (nullable), the permutation and
 * offsets[P+1] (int64). */
int jfx_hash_partition(const jfx_column* keys, int ncols, int64_t n, int num_partitions,
                       int32_t* targets_out, int32_t* perm_out, int64_t* offsets_out,
                       void* workspace, size_t workspace_bytes, void* stream);

/* Learned-CDF partitioned sort of uint64 keys (no counterpart in the
 * reference; its output is exactly the plain radix sort's: sorted keys and
 * the stable int32 permutation).  A 1% strided sample, sorted by the plain
 * radix sort, trains a two-level piecewise-linear model (root line plus 4096
 * leaf lines, least squares) of each key's position.  The predicted
 * position's top bits name a bucket of about 2048 rows; two stable radix
 * passes over the bucket id move (key, row id) into bucket order, and each
 * bucket is then sorted by key inside one CTA (a bucket too large for shared
 * memory by one CTA in global memory, or above 2^20 rows by the plain radix
 * sort).  mode 0: learned, with the plain sort as fallback when the model
 * fails its monotonicity check or more than 4096 buckets are too large for
 * shared memory; mode 1: plain radix sort only.  *learned_used (nullable) is
 * 1 when the learned path produced the result, 0 when the plain sort was
 * asked for or the input is small, and -1 / -3 when the learned path fell
 * back (model check failed / large-bucket list full). */
int jfx_learned_sort(const uint64_t* keys, int64_t n, uint64_t* sorted_keys_out, int32_t* perm_out,
                     int mode, int32_t* learned_used, void* workspace, size_t workspace_bytes,
                     void* stream);

/* Many independent queries in one kernel launch (no host synchronisation,
 * so it can be captured in one CUDA graph).  Query q owns rows
 * [query_offsets[q], query_offsets[q+1]) of keys/values (device int64[nq+1];
 * n = query_offsets[nq], given by the host).  Per query it computes the
 * one-device body of collective_hash_repartition with num_partitions
 * partitions (parallel_algorithms.py:163-182, :213-214: partition
 * fmix32(key) % P, stable) and SortBasedGroupBy.groupby_aggregate sum and
 * count of the values (:733-803; count in the value dtype):
 *   part_keys_out / part_values_out [n]: rows in partition order per query;
 *   part_offsets_out [nq * (P+1)]: absolute row offsets of each partition;
 *   group_keys_out / group_sums_out / group_counts_out [capacity n]: groups
 *   of query q at [group_offsets_out[q], group_offsets_out[q+1]), keys
 *   ascending.
 * Keys must lie in [0, 2^key_bits); jfx_batch_status reports a violation.
 * One persistent kernel launch does all of it: a device work queue of the
 * queries, largest first, each query's partition, bucket pass and groupby
 * run by one CTA; group sums are accumulated in float64 and rounded once. */
int jfx_batch_partition_groupby(const int32_t* keys, const float* values, const int64_t* query_offsets,
                                int nq, int64_t n, int num_partitions, int key_bits,
                                int32_t* part_keys_out, float* part_values_out,
                                int64_t* part_offsets_out, int32_t* group_keys_out,
                                float* group_sums_out, float* group_counts_out,
                                int64_t* group_offsets_out, void* workspace, size_t workspace_bytes,
                                void* stream);

/* Status of the batched call that last used this workspace (synchronises). */
int jfx_batch_status(void* workspace, size_t workspace_bytes, void* stream);

/* Tuning of this thread's later calls (no counterpart in the reference): the
 * widest radix digit per pass (8..11 bits; passes = ceil(key bits / width)),
 * whether the passes after the first run in two phases (per-tile digit
 * counts and a scan first, then the pass without a look-back; 1, the
 * default) or as single look-back passes (0), and the bound of every
 * device-side wait in microseconds (a decoupled look-back that waits longer
 * on an earlier tile gives up and the call returns JFX_ERR_TIMEOUT; 1..10^7,
 * default 10^6 = 1 s).  jfx_set_tuning(NULL) restores the defaults.  The
 * autotuner (jaxframes_b200/autotune.py) picks values per key dtype, size and
 * skew. */
typedef struct {
  int32_t max_digit_bits;
  int32_t two_phase;
  int32_t spin_limit_us;
  int32_t reserved;
} jfx_tuning;
int jfx_set_tuning(const jfx_tuning* t);
int jfx_get_tuning(jfx_tuning* t);

/* Failure injection for this thread's later calls, to test the error paths
 * without faulting a GPU (no counterpart in the reference).  All zero (or
 * jfx_set_fault(NULL)) injects nothing.
 *   withhold_tile:    >= 1: in every decoupled look-back pass, the tile with
 *                     that ticket never publishes its counts, so the later
 *                     tiles' bounded waits run out and the call returns
 *                     JFX_ERR_TIMEOUT (give a short spin_limit_us);
 *   learned_fallback: -1 / -3: jfx_learned_sort takes that fallback (model
 *                     check failed / large-bucket list full) as if its own
 *                     check had found it; the output is the plain sort's;
 *   fail_workspace:   1: every entry point that takes a workspace reports it
 *                     as too small (JFX_ERR_ALLOC) before launching anything;
 *   withhold_order:   1: the batch kernel never publishes its query order, so
 *                     every CTA's bounded wait runs out, the kernel exits and
 *                     jfx_batch_status returns JFX_ERR_TIMEOUT (give a short
 *                     spin_limit_us). */
typedef struct {
  int32_t withhold_tile;
  int32_t learned_fallback;
  int32_t fail_workspace;
  int32_t withhold_order;
} jfx_fault;
int jfx_set_fault(const jfx_fault* f);

/* Measurement hooks.  No counterpart in the reference, which has no tracing.
 * jfx_launch_count: number of kernels this library has launched so far.
 * jfx_timing_enable(1) clears and starts CUDA-event timing of the radix pass
 * kernels on their launching streams; jfx_timing_read waits for the recorded
 * launches and returns their summed duration, count and algorithmic bytes. */
uint64_t jfx_launch_count(void);
int jfx_timing_enable(int enable);
int jfx_timing_read(double* total_ms, int64_t* launches, double* algo_bytes);

#ifdef __cplusplus
}
#endif

#endif /* JFX_H */
