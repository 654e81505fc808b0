/*
 * ghive_b200.h — C ABI of the B200 (sm_100a) relational-operator library.
 *
 * This is the drop-in boundary for the path GHive offloads from Hive's
 * Filter / GroupBy / MapJoin / ReduceSink operators: filter, hash group-by
 * aggregation, hash equi-join (build + probe) and ORDER BY sort over Hive
 * columnar batches.  Every entry point takes plain pointers and sizes; no
 * C++ or torch type crosses it.  The C++ adapters that keep GHive's operator
 * classes (`FilterPredicate::process`, `GroupByPredicate::gpu_execute`,
 * `BaseJoinPredicate::process`, the Sink sort) sit on top of this header in
 * ghive_b200/csrc/host/ghive_ops.hpp, and the JNI shim that keeps
 * `JNIInterface.GPUProcess` sits on top of those.
 *
 * Reference interfaces replaced (paths inside the GHive project):
 *   gpu_impl/inc/DataFlow/Column.hpp:5-35       ColumnType, Column
 *   gpu_impl/inc/DataFlow/Table.hpp:29-52        in-band NULL sentinels
 *   gpu_impl/inc/Operator/FilterPredicate.hpp:17-58   PredicateMode
 *   gpu_impl/src/Operator/FilterPredicate.cu:434-571  FilterPredicate::process
 *   gpu_impl/src/Operator/FilterOperator.cu:36-93     FilterOperator::clean_data
 *   gpu_impl/inc/Operator/AggregationDesc.hpp:6-37    AggregationType / AggregationDesc
 *   gpu_impl/src/Operator/GroupByPredicate.cu:19-359  GroupByPredicate::gpu_execute
 *   gpu_impl/inc/Operator/BaseJoinPredicate.hpp:11-25 BaseJoinType
 *   gpu_impl/src/Operator/SortMergeJoinPredicate.cu:8-461  join process
 *   gpu_impl/src/Operator/BaseJoinPredicate.cu:4-97   generate_result (payload gather)
 *   gpu_impl/src/Operator/SinkOperator.cu:98-306      Sink ORDER BY sort
 *
 * Conventions
 *   - Every function returns GHB_OK (0) or a GHB_ERR_* code; the message of
 *     the last failure on a context is ghb_last_error(ctx).
 *   - Device entry points are asynchronous on the given stream (a
 *     cudaStream_t passed as void*; NULL = legacy default stream).  Row counts
 *     produced on the device are written to a caller-provided DEVICE int64.
 *     ghb_sync() waits for the stream and reports any device-side error
 *     (look-back timeout, output capacity exceeded) raised since the last sync.
 *   - Entry points suffixed _host take HOST buffers, copy them to the device,
 *     run the operator and copy the result back before returning.
 *   - Row counts are int64 (the reference used uint32, Column.hpp:18).
 */
#ifndef GHIVE_B200_H
#define GHIVE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GHB_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define GHB_OK               0
#define GHB_ERR_INVALID      1   /* bad argument or descriptor; nothing launched */
#define GHB_ERR_OOM          2   /* device scratch could not be allocated        */
#define GHB_ERR_CUDA         3   /* a CUDA runtime call failed                   */
#define GHB_ERR_TIMEOUT      4   /* a bounded device-side wait gave up           */
#define GHB_ERR_CAPACITY     5   /* output buffer too small; required rows known */
#define GHB_ERR_UNSUPPORTED  6   /* valid request outside what the kernels do    */

/* ---- column types: same values as GHive's ColumnType (Column.hpp:5-11) -- */
#define GHB_LONG    0   /* int64  (Hive LongColumnVector.vector)   */
#define GHB_DOUBLE  1   /* double (Hive DoubleColumnVector.vector) */
#define GHB_INT     2   /* int32  (GHive INT column)               */
#define GHB_STRING  3   /* data: UTF-8 bytes; aux: int32 [start,end) per row,
                            start < 0 = NULL (GTable.java:240-257).  As an
                            output column: data holds the int32 [start,end)
                            pairs into the input column's bytes */

/* ---- NULL conventions ---------------------------------------------------- */
#define GHB_NULLS_NONE      0  /* Hive noNulls == true                                   */
#define GHB_NULLS_SENTINEL  1  /* GHive in-band: INT64_MAX / NaN / INT32_MAX (Table.hpp:29-52) */
#define GHB_NULLS_BYTEMAP   2  /* Hive ColumnVector.isNull[]: one byte per row, nonzero = NULL */

/* ---- predicate modes: same values as GHive's PredicateMode
 *      (FilterPredicate.hpp:17-58); semantics of the leaves follow Hive's
 *      FilterColumnCompareScalar / FilterColumnBetween templates: a NULL
 *      operand never passes. ------------------------------------------------ */
#define GHB_FILTER_EQ            0   /* x == a            */
#define GHB_FILTER_LE            1   /* x <= a            */
#define GHB_FILTER_GE            2   /* x >= a            */
#define GHB_FILTER_LT            3   /* x <  a            */
#define GHB_FILTER_GT            4   /* x >  a            */
#define GHB_FILTER_RANGE         5   /* a <  x <  b       */
#define GHB_FILTER_EQ_RANGE      6   /* a <= x <= b (BETWEEN) */
#define GHB_FILTER_NOT_EQ        7   /* x != a            */
#define GHB_FILTER_NOT_RANGE     8   /* x < a || x > b (NOT BETWEEN) */
#define GHB_FILTER_NOT_EQ_RANGE  9   /* x <= a || x >= b  */
#define GHB_FILTER_NOT_NULL     10   /* x IS NOT NULL     */
#define GHB_FILTER_AND          11
#define GHB_FILTER_OR           12

/* ---- aggregation types: same values as GHive's AggregationType
 *      (AggregationDesc.hpp:6-25).  Result types follow Hive's UDAFs:
 *      SUM(int/long) -> int64 with silent wrap; SUM(double) -> double;
 *      AVG -> double (sum kept in double, VectorUDAFAvg.txt:56-71);
 *      MIN/MAX -> input type; CNT -> int64 (COUNT(*) when col < 0). ------- */
#define GHB_AGG_SUM  0
#define GHB_AGG_MAX  1
#define GHB_AGG_MIN  2
#define GHB_AGG_AVG  3
#define GHB_AGG_CNT  4

/* ---- join types: same values as GHive's BaseJoinType (BaseJoinPredicate.hpp:11-25) */
#define GHB_INNER_JOIN       0
#define GHB_LEFT_OUTER_JOIN  1   /* probe side is the left (preserved) side */
#define GHB_LEFT_SEMI_JOIN   4

/* ---- sort orders (SinkOperator "sort order: +-"; null order 'a'/'z') ---- */
#define GHB_ASC   0
#define GHB_DESC  1
#define GHB_NULLS_DEFAULT 0  /* Hive default: ASC -> NULLS FIRST, DESC -> NULLS LAST */
#define GHB_NULLS_FIRST   1
#define GHB_NULLS_LAST    2

/* An input column.  `data` holds n values of `type`.  For GHB_STRING, `data`
 * is the char blob and `aux` the int32 [start,end) pair array (GHive's
 * Column::data_ptr_aux); -1,-1 is NULL. */
typedef struct ghb_column {
  int32_t type;
  int32_t null_mode;
  const void* data;
  const uint8_t* is_null;   /* used when null_mode == GHB_NULLS_BYTEMAP */
  const void* aux;          /* GHB_STRING only */
  int64_t n;
} ghb_column;

/* An output column with room for the capacity the call states.  `is_null`
 * may be NULL when the caller knows no output value can be NULL; an
 * aggregate that can be NULL (SUM/AVG/MIN/MAX over an all-NULL group)
 * then writes the GHive sentinel of its type instead. */
typedef struct ghb_out_column {
  int32_t type;
  int32_t reserved;
  void* data;
  uint8_t* is_null;
} ghb_out_column;

/* One node of a predicate tree (GHive FilterPredicate, FilterPredicate.hpp:60-117).
 * Leaves compare column `col` with the literals, or with column `col2` when
 * col2 >= 0 (column-vs-column; only the binary compare modes).  A literal is
 * read as double when lit_is_double != 0, else as int64; the comparison runs
 * in double when either side is double (Java binary numeric promotion), else
 * in int64.  A leaf on a STRING column compares with the byte strings
 * lit_s[k] (lit_s_len[k] bytes, not NUL-terminated; at most
 * GHB_MAX_PRED_STR_BYTES over a tree) as Hive's StringExpr.compare does
 * (storage-api/.../StringExpr.java:37-47: unsigned bytes, then length; GHive's
 * filter_str_unary_* functors, FilterPredicate.hpp:416-683, compare signed
 * chars instead).  AND/OR nodes name two children by node index. */
typedef struct ghb_pred_node {
  int32_t mode;
  int32_t col;
  int32_t col2;
  int32_t lit_is_double;
  int32_t child[2];
  int64_t lit_i[2];
  double lit_d[2];
  const char* lit_s[2];
  int32_t lit_s_len[2];
} ghb_pred_node;
#define GHB_MAX_PRED_STR_BYTES 512

typedef struct ghb_predicate {
  int32_t n_nodes;   /* <= GHB_MAX_PRED_NODES */
  int32_t root;
  const ghb_pred_node* nodes;
} ghb_predicate;
#define GHB_MAX_PRED_NODES 32

/* GHive AggregationDesc{type, index}; col < 0 with GHB_AGG_CNT is COUNT(*). */
typedef struct ghb_agg_desc {
  int32_t type;
  int32_t col;
} ghb_agg_desc;

/* Tuning knobs (zero = library default / autotuned choice). */
typedef struct ghb_groupby_cfg {
  int32_t block_threads;      /* threads per CTA                              */
  int32_t smem_slots;         /* shared-memory pre-aggregation slots per CTA;
                                 -1 disables the shared stage                 */
  int32_t global_slots_log2;  /* log2 of the global table size (0 = from max_groups) */
  int32_t ctas_per_sm;        /* persistent CTAs per SM                       */
  int64_t max_groups;         /* capacity hint = output capacity              */
  int32_t tile_rows;          /* rows per shared-memory tile: the block size
                                 or twice it; 0 = chosen with the stages      */
  int32_t nstages;            /* tile stages, 2..8; 0 = enough for ~64 KB of
                                 copies in flight                             */
} ghb_groupby_cfg;

typedef struct ghb_join_cfg {
  float load_factor;          /* build table fill, default 0.5               */
  int32_t l2_persist;         /* 1: pin the table in L2 with an access-policy window */
  int32_t block_threads;
} ghb_join_cfg;

typedef struct ghb_sort_cfg {
  int32_t digit_bits;         /* radix digit width (8..12), 0 = default      */
  int32_t block_threads;
  int32_t items_per_thread;
} ghb_sort_cfg;

typedef struct ghb_ctx ghb_ctx;
typedef struct ghb_join_table ghb_join_table;

/* ---- context ---------------------------------------------------------- */
/* Creates a context on `device`.  The context owns a growable device scratch
 * arena (hash tables, look-back state); `arena_bytes` pre-reserves it
 * (0 = grow on demand).  Replaces the process-global state GHive keeps in
 * Parser.cu:16-20; contexts are independent and may be used from different
 * host threads (one thread per context at a time). */
int32_t ghb_ctx_create(int32_t device, int64_t arena_bytes, ghb_ctx** out);
int32_t ghb_ctx_destroy(ghb_ctx* ctx);
const char* ghb_last_error(const ghb_ctx* ctx);
int32_t ghb_abi_version(void);
/* Waits for `stream` and returns the first device-side error recorded on the
 * context since the previous ghb_sync (GHB_OK if none), then clears it. */
int32_t ghb_sync(ghb_ctx* ctx, void* stream);
/* Number of kernels the context launched since creation. */
int64_t ghb_kernel_launches(const ghb_ctx* ctx);
/* Bound of the decoupled look-back waits (filter, join probe offsets, sort
 * passes) of this context's later launches: a CTA that polls an earlier,
 * not yet published tile `polls` times gives up, raises GHB_ERR_TIMEOUT
 * (reported by ghb_sync) and returns; its results are then invalid, but
 * every write stays inside the caller's buffers.  polls <= 0 restores the
 * default (2^21 polls, about a second).  No counterpart in the reference,
 * whose waits are inside Thrust; a small bound lets a test reach the
 * timeout path on purpose. */
int32_t ghb_ctx_set_spin_limit(ghb_ctx* ctx, int32_t polls);

/* Per-call tracing.  Every operator entry point opens an NVTX range named for
 * the operator (seen by Nsight tools when one is attached).  With a log open,
 * each call of this context also appends one JSON line to `path`:
 *   level 1: {"op", "device", "rows", "bytes", "host_us", "status"}: rows and
 *            the algorithmic input bytes of the call, and its host-side time
 *            (the enqueue of an asynchronous call; all of a host-buffer or
 *            plan call);
 *   level 2: the call is bracketed by events on its stream and waited for,
 *            adding "device_us", "gbs" and, with peak_gbs > 0,
 *            "roofline_frac" = gbs / peak_gbs.  For measurement only: it
 *            synchronises every call and must not be used under stream capture.
 * path NULL or level 0 closes the log.  ghb_ctx_create opens one when the
 * environment sets GHB_LOG=<path> (GHB_LOG_LEVEL, GHB_LOG_PEAK_GBS). */
int32_t ghb_ctx_set_log(ghb_ctx* ctx, const char* path, int32_t level, double peak_gbs);

/* ---- filter (F1) -------------------------------------------------------
 * Replaces FilterPredicate::process (FilterPredicate.cu:434-571) followed by
 * FilterOperator::clean_data (FilterOperator.cu:36-93): evaluates the
 * predicate tree on `cols` and writes the selected rows of the columns listed
 * in `proj` (indices into cols) to `out[0..nproj)`, in input order.  The
 * inputs are not modified (the reference compacted them in place).  STRING
 * columns may be predicate leaves and projections (a projected STRING row
 * is its [start,end) pair into the input's bytes, GPU memory read only).
 * d_out_rows (device int64) receives the number of selected rows.  Rows
 * beyond out_capacity are counted but not written; ghb_sync then returns
 * GHB_ERR_CAPACITY. */
int32_t ghb_filter(ghb_ctx* ctx, const ghb_predicate* pred,
                   const ghb_column* cols, int32_t ncols,
                   const int32_t* proj, int32_t nproj,
                   ghb_out_column* out, int64_t out_capacity,
                   int64_t* d_out_rows, void* stream);

/* ---- fused filter + hash group-by (G1/G2) -----------------------------
 * Replaces GroupByPredicate::gpu_execute (GroupByPredicate.cu:19-359) fed by
 * the filter above; the predicate (nullable) is evaluated inside the
 * aggregation kernel so no filtered table is materialised.  Output columns:
 * out[0..nkeys) = group keys, out[nkeys..nkeys+naggs) = aggregates, one row
 * per group in unspecified order (Hive's HashMap order is unspecified too).
 * With nkeys == 0 the result is one row (Hive's global aggregate, also on an
 * empty input).  d_out_groups (device int64) receives the group count.
 * Several key columns (GroupByPredicate.cu:24-105 sorts by all of them) are
 * packed into one 64-bit key per row after one read of their ranges (a
 * stream synchronisation); key tuples whose ranges need more than 63 bits
 * together are grouped by the row of each tuple's first occurrence (a device
 * hash table of the tuples).  STRING key columns are
 * first mapped to the row of their value's first occurrence on the device
 * (GroupByPredicate.hpp:75-101 compares the bytes); a STRING key's output is
 * [start,end) pairs into the key column's own bytes.  STRING columns may be
 * predicate leaves too, not aggregate inputs. */
int32_t ghb_filter_groupby(ghb_ctx* ctx, const ghb_predicate* pred,
                           const ghb_column* cols, int32_t ncols,
                           const int32_t* key_cols, int32_t nkeys,
                           const ghb_agg_desc* aggs, int32_t naggs,
                           ghb_out_column* out, int64_t out_capacity,
                           int64_t* d_out_groups,
                           const ghb_groupby_cfg* cfg, void* stream);

/* ---- hash join (J1 build, J2 probe) ------------------------------------
 * Replaces the sort + CPU merge of SortMergeJoinPredicate::process
 * (SortMergeJoinPredicate.cu:8-461) and the host gather of
 * BaseJoinPredicate::generate_result (BaseJoinPredicate.cu:4-97) with a
 * device hash join on one LONG or INT key.  Like Hive's hash map, which
 * stores each build row's retained values with its key
 * (VectorMapJoinFastLongHashMap.java:71-84), the table holds the build
 * payload columns: the first build row of every key is copied into its slot
 * (up to two 8-byte non-BYTEMAP payloads), the others are read from the
 * build_payload columns, which must stay valid until the table is freed.
 * The table stays resident on the device until ghb_join_table_free, so one
 * build serves many probes (a broadcast map-join small table).  NULL build
 * keys are not inserted; NULL probe keys never match.  At most
 * GHB_MAX_JOIN_PAYLOAD build payloads (and as many probe payloads per probe). */
#define GHB_MAX_JOIN_PAYLOAD 16
int32_t ghb_join_build(ghb_ctx* ctx, const ghb_column* build_key,
                       const ghb_column* build_payload, int32_t n_build_payload,
                       const ghb_join_cfg* cfg, ghb_join_table** out,
                       void* stream);
int32_t ghb_join_table_free(ghb_ctx* ctx, ghb_join_table* table);
/* Rows stored and the largest number of build rows sharing one key
 * (valid after ghb_sync of the build stream). */
int32_t ghb_join_table_info(ghb_ctx* ctx, const ghb_join_table* table,
                            int64_t* rows, int64_t* max_dup, int64_t* slots);

/* Probes `probe_key` against `table` (join_type GHB_INNER_JOIN,
 * GHB_LEFT_SEMI_JOIN or GHB_LEFT_OUTER_JOIN).  Each output row is one
 * (probe row, build row) pair, in probe-row order.  Written per output row,
 * each optional (NULL to skip):
 *   out_probe_rowid[i]  probe row index (int32)
 *   out_build_rowid[i]  build row index (int32; -1 for an outer-join miss)
 *   out_build[j]        the table's build payload j at the build row
 *                       (NULL in is_null / sentinel for an outer miss);
 *                       an array of the table's n_build_payload columns
 *   out_probe[j]        probe_payload[j] gathered at the probe row
 * d_out_rows (device int64) receives the number of output rows. */
int32_t ghb_join_probe(ghb_ctx* ctx, const ghb_join_table* table,
                       const ghb_column* probe_key, int32_t join_type,
                       ghb_out_column* out_build,
                       const ghb_column* probe_payload, int32_t n_probe_payload,
                       ghb_out_column* out_probe,
                       int32_t* out_probe_rowid, int32_t* out_build_rowid,
                       int64_t out_capacity, int64_t* d_out_rows, void* stream);

/* ---- ORDER BY sort (S1) -------------------------------------------------
 * Replaces the Sink sort (SinkOperator.cu:153-286): a stable sort of n rows
 * by the key columns in Hive's BinarySortable order (BinarySortableSerDe.java:
 * 921-960: signed integers and IEEE doubles in numeric order, per-key ASC/DESC
 * and NULLS FIRST/LAST).  Writes the sorted key columns to out_keys and the
 * payload columns, permuted the same way, to out_payload; out_rowid (nullable,
 * int32) receives the permutation.  Ties keep input order.  A STRING key
 * sorts by unsigned bytes, then length (StringExpr.java:37-47), as the
 * tuple of its 8-byte parts and its length (one read finds the longest
 * string; at most 8 key parts in all); its output is [start,end) pairs into
 * the key column's bytes.  Payloads are fixed-width. */
int32_t ghb_sort(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                 const int32_t* null_orders, int32_t nkeys,
                 const ghb_column* payload, int32_t npayload,
                 ghb_out_column* out_keys, ghb_out_column* out_payload,
                 int32_t* out_rowid, const ghb_sort_cfg* cfg, void* stream);

/* ---- fused filter + group-by without allocation -------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * a task whose device memory is all reserved by another allocator, or code
 * that must not risk the device-wide synchronisation an allocation may
 * imply.  Same operator and arguments as ghb_filter_groupby (device columns,
 * device outputs, device group count), but no context: the hash table and the
 * device status word live in a file-scope __device__ array of
 * GHB_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; nothing is allocated or freed.  The table needs
 * (C + 2) * 8 * R + 16 + C / 8 bytes, with
 * C = next_pow2(max(2 * max_groups + 1, 64)) and R = 1 + accumulator words
 * (one accumulator word per COUNT/SUM/MIN/MAX state, two per double SUM/AVG,
 * plus COUNT(*)), R rounded up to 2, 4, 8, 16 or 24 when C > 2^17; a call
 * that would need more than the array holds returns GHB_ERR_CAPACITY before
 * launching.  About 60,000 groups fit with the fact-table aggregates.
 * The first call on a device is its set-up: it looks up the array's device
 * address and loads the array and every kernel the call launches (CUDA
 * loads code lazily, and loading may allocate device memory).  Make that
 * first call before handing the device's memory to another allocator and
 * before any stream capture; later calls load and allocate nothing.  The
 * looked-up address is kept for the life of the process (it assumes no
 * cudaDeviceReset).  Each call clears the part of the
 * array it uses, runs on `stream`, waits for it and returns the device
 * status (GHB_ERR_CAPACITY for a short output).  Calls share the one array:
 * calls that overlap on the GPU (other streams, other host threads) race and
 * corrupt each other's tables. */
#define GHB_NOALLOC_SCRATCH_BYTES (8u << 20)
int32_t ghb_filter_groupby_noalloc(const ghb_predicate* pred,
                                   const ghb_column* cols, int32_t ncols,
                                   const int32_t* key_cols, int32_t nkeys,
                                   const ghb_agg_desc* aggs, int32_t naggs,
                                   ghb_out_column* out, int64_t out_capacity,
                                   int64_t* d_out_groups,
                                   const ghb_groupby_cfg* cfg, void* stream);

/* ---- batched filter + group-by -------------------------------------------
 * GHive runs one GroupByPredicate::gpu_execute per Tez task
 * (GroupByOperator::execute, gpu_impl/src/Operator/GroupByOperator.cu:
 * 101-130), one launch sequence per split.  A batch runs many instances of
 * one operator signature (the same key column, aggregates and column types;
 * each instance with its own columns, row count, predicate literals, output
 * columns and group count) in one persistent fold kernel and one finalize,
 * captured once in a CUDA graph.  ghb_batch_groupby_create validates the
 * instances, optionally autotunes (CTA size per batch; shared-table size,
 * load factor and warp combining per size class of rows x groups, timed on
 * the class's largest instance), sizes one global table per instance and
 * captures the launches; it synchronises `stream`.  ghb_batch_launch
 * replays them on `stream`: every instance's output columns and
 * d_out_groups[i] are rewritten from the current contents of its columns
 * (the same device addresses as at creation).  Results are those of
 * ghb_filter_groupby on each instance alone.  Errors raised on the device
 * (GHB_ERR_CAPACITY when an instance has more groups than max_groups allows
 * or than its out_capacity) are reported by ghb_sync. */
typedef struct ghb_groupby_instance {
  const ghb_column* cols;      /* ncols device columns of one length        */
  const ghb_predicate* pred;   /* NULL: every row passes                    */
  ghb_out_column* out;         /* nkeys + naggs device output columns       */
  int64_t out_capacity;
  int64_t max_groups;          /* groups expected; 0 = out_capacity         */
} ghb_groupby_instance;

typedef struct ghb_batch_cfg {
  int32_t autotune;            /* 1: time candidate settings at creation    */
  int32_t block_threads;       /* 512 or 1024; 0 = tuned, else 1024         */
  int32_t smem_slots;          /* 0 = tuned / automatic, -1 = no shared table */
  float load_factor;           /* 0 = tuned / 0.5                           */
  int32_t use_graph;           /* 0: plain launches; otherwise a CUDA graph */
} ghb_batch_cfg;

typedef struct ghb_batch ghb_batch;
int32_t ghb_batch_groupby_create(ghb_ctx* ctx, const ghb_groupby_instance* inst,
                                 int32_t ninst, int32_t ncols,
                                 const int32_t* key_cols, int32_t nkeys,
                                 const ghb_agg_desc* aggs, int32_t naggs,
                                 int64_t* d_out_groups, const ghb_batch_cfg* cfg,
                                 void* stream, ghb_batch** out);
int32_t ghb_batch_launch(ghb_batch* batch, void* stream);
/* The settings the batch runs with (JSON text: block size, grid, chunks and
 * per size class the shared slots, load factor and measured ns per row). */
int32_t ghb_batch_describe(const ghb_batch* batch, char* buf, int64_t len);
int32_t ghb_batch_destroy(ghb_batch* batch);

/* ---- specialised group-by kernels ----------------------------------------
 * No counterpart in the reference.  A fused filter + group-by call compiles
 * (NVRTC, sm_100a) and caches a fold kernel specialised for its signature:
 * the used columns' types and NULL modes, the predicate tree's shape, the key
 * column and the aggregates; literal values stay run-time parameters.  The
 * cache is per process and on disk ($GHB_JIT_CACHE, default
 * ~/.cache/ghive_b200/jit); GHB_JIT=0 in the environment runs the generic
 * kernel instead.  These two functions need no GPU: one writes the kernel
 * source a call would compile (batch != 0: the batched fold), the other
 * compiles a source and reports the cubin size and the compiler log, to
 * check or pre-build kernels ahead of the first call. */
int32_t ghb_jit_groupby_source(const ghb_predicate* pred, const ghb_column* cols,
                               int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                               const ghb_agg_desc* aggs, int32_t naggs, int32_t batch,
                               char* buf, int64_t len);
int32_t ghb_jit_compile_source(const char* source, int64_t* cubin_bytes, char* log,
                               int64_t len);

/* ---- serving: concurrent operator requests ------------------------------
 * GHive's JNI entry point (GPUProcess, gpu_impl/src/ghive_JNIInterface.cu:
 * 13-340) runs one Tez task's plan alone: every call re-uploads its inputs,
 * rebuilds its join tables and owns the GPU until it returns.  A server is
 * long-lived and shared by many host threads (Hive tasks): a request is
 * queued on submit and admitted as soon as one of `slots` execution slots is
 * free and its HBM footprint (outputs + working memory) fits the budget;
 * admitted requests run concurrently, one CUDA stream and one context per
 * slot, so a request that arrives while others are on the GPU overlaps with
 * them (continuous batching).  Join build tables registered with the server
 * stay resident across requests.  Inputs are device columns that must stay
 * valid until the request is done; outputs are device buffers owned by the
 * server until ghb_server_release.  Results are those of the plain operator
 * on the same inputs.  All functions are thread-safe. */
#define GHB_OP_FILTER 0
#define GHB_OP_GROUPBY 1
#define GHB_OP_JOIN_PROBE 2
#define GHB_OP_SORT 3
#define GHB_MAX_RESULT_COLS 16

typedef struct ghb_server_cfg {
  int32_t slots;               /* requests on the device at once (0 = 8)    */
  int32_t reserved;
  int64_t hbm_budget;          /* bytes admitted at once (0 = 40% of free);
                                  mapped into the server's memory pool when
                                  it is created, so serving never grows it */
} ghb_server_cfg;

typedef struct ghb_request {
  int32_t op;                  /* GHB_OP_*                                    */
  int32_t ncols;
  const ghb_column* cols;      /* FILTER/GROUPBY inputs; JOIN_PROBE: cols[0] =
                                  probe key; SORT: keys then payload          */
  const ghb_predicate* pred;   /* FILTER, GROUPBY (NULL = all rows)           */
  const int32_t* idx;          /* FILTER: projection (NULL = all columns);
                                  GROUPBY: key columns                        */
  int32_t nidx;
  int32_t naggs;               /* GROUPBY                                     */
  const ghb_agg_desc* aggs;
  int64_t max_groups;          /* GROUPBY: output capacity in groups          */
  int32_t table;               /* JOIN_PROBE: id from ghb_server_add_join_table */
  int32_t join_type;
  int32_t nkeys;               /* SORT: leading key columns                   */
  int32_t want_rowid;          /* SORT: emit input row ids; JOIN_PROBE: also
                                  emit build row ids                          */
  const int32_t* orders;       /* SORT (NULL = all ASC)                       */
  const int32_t* null_orders;  /* SORT (NULL = Hive defaults)                 */
} ghb_request;

typedef struct ghb_result {
  int32_t status;              /* GHB_OK or the operator's error              */
  int32_t ncols;
  ghb_out_column cols[GHB_MAX_RESULT_COLS];  /* FILTER: projected columns;
                                  GROUPBY: keys then aggregates; JOIN_PROBE:
                                  the table's payload columns; SORT: keys
                                  then payload                                */
  int32_t* rowid;              /* JOIN_PROBE: probe row ids; SORT: row ids    */
  int32_t* rowid2;             /* JOIN_PROBE: build row ids (want_rowid)      */
  int64_t rows;                /* rows (groups) in the outputs                */
  int64_t submit_ns;           /* CLOCK_MONOTONIC: submitted, admitted, done  */
  int64_t admit_ns;
  int64_t done_ns;
  int64_t launched_ns;         /* the operator's launches had all returned   */
  int32_t slot;                /* the slot that ran it                        */
  int32_t reserved;
} ghb_result;

typedef struct ghb_server ghb_server;
int32_t ghb_server_create(int32_t device, const ghb_server_cfg* cfg, ghb_server** out);
/* Builds a join table on the device and keeps it (with its payload columns,
 * which must stay valid) until the server is destroyed. */
int32_t ghb_server_add_join_table(ghb_server* server, const ghb_column* build_key,
                                  const ghb_column* payload, int32_t npayload,
                                  float load_factor, int32_t* table_id);
int32_t ghb_server_submit(ghb_server* server, const ghb_request* req, uint64_t* ticket);
/* Waits until the request is done and copies its result. */
int32_t ghb_server_wait(ghb_server* server, uint64_t ticket, ghb_result* out);
/* Frees the request's outputs and its share of the budget. */
int32_t ghb_server_release(ghb_server* server, uint64_t ticket);
int32_t ghb_server_stats(ghb_server* server, int64_t* completed, int64_t* running,
                         int64_t* queued, int64_t* bytes_admitted);
const char* ghb_server_last_error(ghb_server* server);
int32_t ghb_server_destroy(ghb_server* server);

/* ---- GHive's JNI input and output, and a vertex's operator chain --------
 * ghb_gtables is GHive's GTables object (ghive/GTables.java:13-31) with its
 * fields read by the JNI shim (GetObjectField, GetIntArrayElements,
 * GetDirectBufferAddress): per input table its column types (0 long,
 * 1 double, 2 int, 3 string), row count, key count and vertex name, and the
 * columns as direct buffers, concatenated by type over the tables in table
 * order.  The buffers are the JVM's, valid during the call, and read only. */
typedef struct ghb_gtables {
  int32_t ntables;
  const int32_t* ncols;                /* types[t].length                     */
  const int32_t* const* types;         /* types[t][c]                         */
  const int32_t* row_cnt;              /* rowCnt[t]                           */
  const int32_t* key_cnt;              /* keyCnt[t]                           */
  const char* const* vertex_name;      /* vertexName[t]; NULL entry: missing  */
  int32_t nlong;
  const void* const* long_cols;        /* longCols[i]: int64 little-endian    */
  int32_t ndouble;
  const void* const* double_cols;      /* doubleCols[i]                       */
  int32_t nint;
  const void* const* int_cols;         /* intCols[i]: int32                   */
  int32_t nstring;
  const void* const* string_cols;      /* stringCols[i]: UTF-8 bytes          */
  const void* const* string_idx_cols;  /* stringIdxCols[i]: int32 [start,end) per row */
} ghb_gtables;

/* Input table `table`'s columns, in its types[] order, as descriptors over
 * the JVM's buffers (no copy; NULLs are GHive's sentinels, GTable.java:
 * 38-40): each column takes the next buffer of its type not taken by an
 * earlier column or table, as GPUProcess does (ghive_JNIInterface.cu:
 * 132-201).  GHB_ERR_INVALID when the table is missing (NULL vertex name),
 * a type's buffers run out or more than `cap` columns would be written. */
int32_t ghb_gtables_table(const ghb_gtables* in, int32_t table, ghb_column* cols,
                          int32_t cap, int32_t* ncols, int64_t* rows);

/* One operator of a vertex's chain (GHive's operator tree of one vertex,
 * Parser.cu:675 root_op->execute(), run here as a chain).  Column indices
 * refer to the table the previous operator produced (the input table for
 * the first). */
typedef struct ghb_plan_op {
  int32_t op;                  /* GHB_OP_FILTER / GROUPBY / JOIN_PROBE / SORT */
  int32_t join_type;           /* JOIN_PROBE                                   */
  const ghb_predicate* pred;   /* FILTER (NULL: a projection alone, which
                                  selects columns without copying them)       */
  const int32_t* idx;          /* FILTER: projection (NULL = all columns);
                                  GROUPBY: key columns; SORT: key columns;
                                  JOIN_PROBE: the k probe key columns, then
                                  the k build key columns of the build table
                                  (k > 1: the tuples are packed into one key,
                                  63 bits at most; a STRING key column of both
                                  sides is first mapped to ids equal exactly
                                  when the strings are)                        */
  int32_t nidx;
  int32_t naggs;               /* GROUPBY                                      */
  const ghb_agg_desc* aggs;
  int64_t max_groups;          /* GROUPBY: output capacity (0 = rows)         */
  const int32_t* orders;       /* SORT (NULL = all ASC)                        */
  const int32_t* null_orders;  /* SORT (NULL = Hive's defaults)                */
  int32_t build_table;         /* JOIN_PROBE: input table of the build side    */
  int32_t nbuild_keep;         /* JOIN_PROBE: build columns appended to the
                                  output, after the probe table's columns     */
  const int32_t* build_keep;
} ghb_plan_op;

/* The final table, host-side, grouped the way GPUResult holds it
 * (GPUResult.java:29-39, built at ghive_JNIInterface.cu:217-340): column i
 * has types[i], data[i] (NULLs as GHive's sentinels) and is_null[i]
 * (NULL: no NULL map), and sequence[i] is its index in the concatenation
 * long || double || int || string of GPUResult's arrays.  A STRING column's
 * data[i] is its int32 [start,end) pairs (-1,-1 = NULL) into str_bytes[i],
 * its rows' UTF-8 bytes packed in row order (str_nbytes[i] of them); it has
 * no NULL map.  The arrays are host memory owned by the library until
 * ghb_plan_result_free. */
typedef struct ghb_plan_result {
  int32_t ncols;
  int32_t types[GHB_MAX_RESULT_COLS];
  void* data[GHB_MAX_RESULT_COLS];
  uint8_t* is_null[GHB_MAX_RESULT_COLS];
  int32_t sequence[GHB_MAX_RESULT_COLS];
  int64_t rows;
  int32_t n_long, n_double, n_int, n_string;
  uint8_t* str_bytes[GHB_MAX_RESULT_COLS];
  int64_t str_nbytes[GHB_MAX_RESULT_COLS];
} ghb_plan_result;

/* Runs `nops` operators on input table `input` of `in`: the table's columns
 * are copied to the device once, every operator's output stays on the device
 * as the next one's input (GHive copied each operator's input in and output
 * back, FilterOperator.cu:53-89, GroupByPredicate.cu:39-91), a JOIN_PROBE
 * builds its hash table from another input table, and only the final table
 * is copied back into `out`.  STRING columns (stringCols with their
 * stringIdxCols) travel as their pairs into bytes copied once: they may be
 * predicate leaves and projections, group-by and sort keys, join keys and
 * payloads of either side, not aggregate inputs.  Synchronous; the
 * context's own stream. */
int32_t ghb_run_plan(ghb_ctx* ctx, const ghb_gtables* in, int32_t input,
                     const ghb_plan_op* ops, int32_t nops, ghb_plan_result* out);
int32_t ghb_plan_result_free(ghb_plan_result* result);

/* ---- host-buffer entry points (end-to-end) -------------------------------
 * Same operators with every column in HOST memory (pageable or pinned).
 * These copy the inputs in, run the operator, copy the result out and
 * synchronise, like one GHive operator call on host `Column`s.  The row
 * count is returned through the host int64 *out_rows. */
/* With every host buffer pinned (or registered) and two chunks of rows or
 * more (about n/12 rows each, 512Ki to 8Mi), the filter runs in chunks whose
 * copies in and out overlap each other and the kernels; the output is the
 * same.  An output capacity below the row count returns GHB_ERR_CAPACITY
 * with the full count in *out_rows (the first out_capacity rows may have
 * been written). */
int32_t ghb_filter_host(ghb_ctx* ctx, const ghb_predicate* pred,
                        const ghb_column* cols, int32_t ncols,
                        const int32_t* proj, int32_t nproj,
                        ghb_out_column* out, int64_t out_capacity,
                        int64_t* out_rows);
int32_t ghb_filter_groupby_host(ghb_ctx* ctx, const ghb_predicate* pred,
                                const ghb_column* cols, int32_t ncols,
                                const int32_t* key_cols, int32_t nkeys,
                                const ghb_agg_desc* aggs, int32_t naggs,
                                ghb_out_column* out, int64_t out_capacity,
                                int64_t* out_groups, const ghb_groupby_cfg* cfg);
int32_t ghb_hash_join_host(ghb_ctx* ctx, const ghb_column* build_key,
                           const ghb_column* probe_key, int32_t join_type,
                           const ghb_column* build_payload, int32_t n_build_payload,
                           ghb_out_column* out_build,
                           const ghb_column* probe_payload, int32_t n_probe_payload,
                           ghb_out_column* out_probe,
                           int32_t* out_probe_rowid, int32_t* out_build_rowid,
                           int64_t out_capacity, int64_t* out_rows,
                           const ghb_join_cfg* cfg);
int32_t ghb_sort_host(ghb_ctx* ctx, const ghb_column* keys, const int32_t* orders,
                      const int32_t* null_orders, int32_t nkeys,
                      const ghb_column* payload, int32_t npayload,
                      ghb_out_column* out_keys, ghb_out_column* out_payload,
                      int32_t* out_rowid, const ghb_sort_cfg* cfg);

#ifdef __cplusplus
}
#endif
#endif /* GHIVE_B200_H */
