/*
 * qm_gpu.h — C ABI of the B200 filter -> hash GROUP BY aggregate path.
 *
 * This is the drop-in boundary that replaces QueryMode's per-batch WASM calls
 * and JS aggregation on the `.filter().groupBy()` / `.sql("... GROUP BY ...")`
 * path.  Every entry point below names the reference interface it replaces.
 * Reference paths are relative to the QueryMode repository root.
 *
 * Conventions (mirroring the WASM boundary, src/wasm-engine.ts:21-187, and the
 * native Node ABI, wasm/src/nodejs.zig:20-40):
 *   - every function returns an int status (QM_OK == 0); on failure the
 *     context keeps a message readable with qm_ctx_last_error();
 *   - handles are opaque and explicitly destroyed;
 *   - a context is used by one host thread at a time (the reference keeps one
 *     single-threaded engine per Durable Object, src/wasm-engine.ts:181-186);
 *     distinct contexts may run concurrently;
 *   - there is no CPU fallback: if no CUDA device or the kernel image is
 *     unavailable, qm_ctx_create fails with QM_ERR_NO_DEVICE / QM_ERR_CUDA.
 *
 * Semantics follow the reference's JS operator path (the parity target):
 *   predicates  src/decode.ts:478-578 (coerceCompare, matchesFilter,
 *               rowPassesFilters), op codes src/operators.ts:422-432;
 *   aggregates  src/partial-agg.ts:38-352 (SUM/COUNT/MIN/MAX/AVG state,
 *               update, merge, finalize), group keys src/types.ts:10-18;
 *   batch merge src/operators.ts:1646-1710 (AggregateOperator.next).
 */
#ifndef QM_GPU_H
#define QM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define QM_OK 0
#define QM_ERR_INVALID 1     /* malformed descriptor / argument            */
#define QM_ERR_UNSUPPORTED 2 /* query shape outside the GPU path           */
#define QM_ERR_CUDA 3        /* CUDA runtime error                          */
#define QM_ERR_OOM 4         /* device allocation or HBM budget refused     */
#define QM_ERR_NOT_FOUND 5   /* unknown column name                         */
#define QM_ERR_CAPACITY 6    /* caller-provided output capacity too small   */
#define QM_ERR_TIMEOUT 7     /* a bounded device-side wait gave up          */
#define QM_ERR_NO_DEVICE 8   /* no CUDA device                              */
#define QM_ERR_CANCELLED 9   /* serving: request cancelled before running   */

/* ---- dtypes: QMCB tags (src/columnar.ts:22-33) ------------------------- */
#define QM_F64 0
#define QM_I64 1
#define QM_I32 6
#define QM_F32 7
/* result-only: exact 128-bit two's-complement integer stored as (lo u64,
 * hi i64) pairs; carries SUM over int64 columns, which the reference keeps
 * as an arbitrary-precision BigInt (src/partial-agg.ts:89-95). */
#define QM_I128 64

/* ---- filter ops: src/types.ts:130-133, codes 0-5 as src/operators.ts:422-432 */
#define QM_OP_EQ 0
#define QM_OP_NEQ 1
#define QM_OP_LT 2
#define QM_OP_LTE 3
#define QM_OP_GT 4
#define QM_OP_GTE 5
#define QM_OP_BETWEEN 6     /* inclusive, src/decode.ts:528-534            */
#define QM_OP_NOT_BETWEEN 7 /* src/decode.ts:535-541                       */
#define QM_OP_IS_NULL 8
#define QM_OP_IS_NOT_NULL 9

/* filter value kinds: a JS `number` or a JS `bigint` (FilterOp.value) */
#define QM_VAL_NUMBER 0
#define QM_VAL_BIGINT 1

/* ---- aggregate fns: src/types.ts:137-145 (numeric subset) -------------- */
#define QM_AGG_SUM 0
#define QM_AGG_AVG 1
#define QM_AGG_MIN 2
#define QM_AGG_MAX 3
#define QM_AGG_COUNT 4

/* ---- query flags --------------------------------------------------------- */
/* Emit groups in hash-table order instead of the reference's Map
 * first-seen order (src/partial-agg.ts:320-349).  Saves one sort. */
#define QM_FLAG_UNORDERED 1
/* Evaluate numeric filters the way the scan-time WASM filter does
 * (src/operators.ts:550-666): NULLs read as 0 and int32 thresholds pass
 * through ToInt32.  Default is the JS matchesFilter semantics. */
#define QM_FLAG_WASM_SCAN_SEMANTICS 2
/* Float SUM / AVG independent of the order rows are added in: each finite
 * cell becomes an exact 128-bit fixed-point integer (units of 2^-k below the
 * column's largest |x|, taken from its statistics) and the integers are
 * summed, so the same query gives bit-identical sums on every run, alone or
 * batched, whatever the launch shape.  The result is the exact sum of the
 * cells rounded once (each cell off by at most 2^-(126 - log2 rows) of the
 * column's largest |x|); NaN / Infinity cells follow the reference's
 * sequential sum.  The reference's own sum is sequential in row order
 * (src/partial-agg.ts:77), which a parallel sum matches only to rounding.
 * Registered tables only (qm_query_run, batches, servers): streamed batches
 * and qm_query_run_noalloc return QM_ERR_UNSUPPORTED. */
#define QM_FLAG_DETERMINISTIC 4

typedef struct qm_ctx qm_ctx;
typedef struct qm_table qm_table;
typedef struct qm_agg qm_agg;
typedef struct qm_result qm_result;

/* One input column.  `null_bitmap` follows QMCB: bit (row & 7) of byte
 * (row >> 3) set = NULL (src/columnar.ts:752-754).  With on_device == 0 the
 * library copies host memory into HBM it owns; with on_device == 1 `data` and
 * `null_bitmap` are device pointers of the context's device, borrowed (not
 * freed) and read in place. */
typedef struct {
  const char *name;
  int32_t dtype;
  int32_t on_device;
  const void *data;
  const uint8_t *null_bitmap;
} qm_column;

/* A JS filter value: `number` (kind QM_VAL_NUMBER, in `num`) or `bigint`
 * (kind QM_VAL_BIGINT, in `big`). */
typedef struct {
  int32_t kind;
  int32_t reserved;
  double num;
  int64_t big;
} qm_value;

/* FilterOp {column, op, value} (src/types.ts:130-134).  BETWEEN uses
 * value (low) and value2 (high). */
typedef struct {
  const char *column;
  int32_t op;
  int32_t reserved;
  qm_value value;
  qm_value value2;
} qm_filter;

/* AggregateOp {fn, column, alias} (src/types.ts:137-145); column "*" is
 * COUNT(*).  A NULL alias means the reference default `${fn}_${column}`
 * (src/partial-agg.ts:136-138). */
typedef struct {
  int32_t fn;
  int32_t reserved;
  const char *column;
  const char *alias;
} qm_aggregate;

/* The filter/groupBy/aggregates part of QueryDescriptor
 * (src/client.ts:1254-1277).  OR groups (QueryDescriptor.filterGroups) are
 * flattened: group g owns or_group_sizes[g] consecutive entries of
 * or_filters.  The row passes if every `filters` entry passes and, when
 * n_or_groups > 0, every entry of at least one group passes
 * (src/decode.ts:558-578). */
typedef struct {
  const qm_filter *filters;
  int32_t n_filters;
  int32_t n_or_groups;
  const int32_t *or_group_sizes;
  const qm_filter *or_filters;
  const char *const *group_by;
  int32_t n_group_by;
  int32_t n_aggregates;
  const qm_aggregate *aggregates;
  int32_t flags;
  int32_t reserved;
  /* Post-aggregate ORDER BY / LIMIT / OFFSET on the result rows, as the
   * reference's pipeline applies them after AggregateOperator
   * (src/operators.ts:3116-3128): with order_by and has_limit, TopKOperator's
   * heap (src/operators.ts:1716-1841, ties resolved as its heap does);
   * order_by alone, InMemorySortOperator's stable sort by rowComparator
   * (src/types.ts:26-38: NULL and NaN last); has_limit or offset alone, the
   * first-seen rows [offset, offset + limit).  order_by names an output
   * column (a group key or an aggregate's alias).  Supported by
   * qm_query_run and qm_agg_finish. */
  const char *order_by;
  int32_t order_desc;
  int32_t has_limit;
  int64_t limit;
  int64_t offset;
} qm_query;

/* One output column.  `data` is host memory owned by the result; dtype is
 * QM_I32/QM_I64/QM_F64 or QM_I128 (2 x 8 bytes per row).  `null_bitmap`
 * is NULL or QMCB-style (bit set = NULL: a NULL group key, or an aggregate
 * whose group saw no non-null value, src/partial-agg.ts:109-111). */
typedef struct {
  const char *name;
  int32_t dtype;
  int32_t is_key;
  int64_t n_rows;
  const void *data;
  const uint8_t *null_bitmap;
} qm_result_col;

/* Per-run counters (the reference reports scanMs / bytesRead / wasmExecMs,
 * src/operators.ts:180-182, src/types.ts:262-300). */
typedef struct {
  int64_t rows_scanned;
  int64_t rows_selected;
  int64_t groups;
  int64_t bytes_scanned;  /* algorithmic: rows x widths of referenced columns */
  double device_ms;       /* CUDA-event time of the device work of the run  */
  int32_t strategy;       /* 0 direct-mapped, 1 block-local + global hash,
                             2 global hash only, 3 hash-partitioned          */
  int32_t table_capacity; /* log2 of the group table's slot count           */
  int32_t retries;        /* table regrowths after a capacity overflow      */
  int32_t launches;       /* kernels of this library launched by the run   */
  double scan_ms;         /* CUDA-event time of the fused scan kernel(s)    */
} qm_stats;

/* Launch-shape knobs of the fused scan kernel, chosen by the autotuner
 * (querymode_b200/autotune.py).  Zero / negative fields mean "planner's
 * choice".  No reference counterpart (the WASM engine has no launch shape). */
typedef struct {
  int32_t local_slots;   /* block-local table slots: 0 auto, -1 none, else a power of two */
  int32_t dedupe;        /* warp-level merge of equal keys: -1 auto, 0 off, 1 on */
  int32_t blocks_per_sm; /* resident blocks per SM: 0 auto (occupancy), else a cap */
  int32_t stage_depth;   /* filter-column tiles in flight per warp (bulk async
                            copies into shared memory): <= 0 off, 2..4 */
  int32_t partitioned;   /* 1: partitioned aggregation (survivors written to key
                            partitions, each aggregated in shared memory) for
                            grouped queries whose table exceeds shared memory
                            and which select at least a quarter of the rows;
                            0 (default): the fused scan */
  int32_t reserved;
} qm_tuning;

/* ---- library / context ---------------------------------------------------- */
const char *qm_version(void);

/* Replaces WebAssembly.instantiate + WasmEngine construction
 * (src/wasm-engine.ts:151-187, src/local-executor.ts:85-98).  `device` is a
 * CUDA ordinal; the context owns a stream and a device memory pool. */
int qm_ctx_create(int32_t device, qm_ctx **out);
int qm_ctx_destroy(qm_ctx *ctx);
/* Replaces WasmEngine.getLastError (src/wasm-engine.ts:272-279). */
const char *qm_ctx_last_error(const qm_ctx *ctx);
/* Order the context's device work on a caller's stream (a cudaStream_t of
 * the context's device, e.g. torch.cuda.current_stream().cuda_stream);
 * NULL restores the context's own stream.  No reference counterpart: the
 * WASM engine has no streams; this lets a host framework time or overlap
 * the path with its own work. */
int qm_ctx_set_stream(qm_ctx *ctx, void *stream);
/* Set (tuning != NULL) or clear (NULL) the context's launch-shape knobs. */
int qm_ctx_set_tuning(qm_ctx *ctx, const qm_tuning *tuning);
/* Device blocks of destroyed tables are kept by the context for the next
 * tables of about their size (up to an eighth of the device's memory; given
 * back by this library whenever one of its allocations fails, and at
 * qm_ctx_destroy).  Batch and serving buffers come from the device's
 * stream-ordered memory pool and stay in it when freed.  This frees both
 * now, for a caller whose other allocators need the memory; *released (may
 * be null) receives the table-block bytes freed.  No counterpart in the
 * reference (device memory management). */
int qm_ctx_trim(qm_ctx *ctx, int64_t *released);
/* Device properties the host planner and tests read. */
int qm_ctx_device_info(const qm_ctx *ctx, int32_t *sm_count, int64_t *hbm_bytes);

/* ---- tables ---------------------------------------------------------------- */
/* Register a table of numeric columns resident in HBM.  Replaces the
 * per-page copy into WASM linear memory (src/operators.ts:558-583) and the
 * in-memory table of MaterializedExecutor (src/client.ts:996-1127). */
int qm_table_create(qm_ctx *ctx, int64_t n_rows, int32_t n_cols,
                    const qm_column *cols, qm_table **out);
/* Register a table from one QMCB buffer (src/columnar.ts:438-516).
 * Numeric columns (F64/I64/I32/F32) are uploaded; others are ignored. */
int qm_table_from_qmcb(qm_ctx *ctx, const uint8_t *buf, size_t len,
                       qm_table **out);
int qm_table_destroy(qm_table *table);
int qm_table_num_rows(const qm_table *table, int64_t *out);
/* The table's columns: how many, and column i's name (owned by the table)
 * and dtype.  No counterpart in the reference (inspection and tests). */
int qm_table_num_columns(const qm_table *table, int32_t *out);
int qm_table_column(const qm_table *table, int32_t column, const char **name, int32_t *dtype);

/* ---- one-shot query over a registered table ---------------------------- */
/* filter -> GROUP BY -> finalize over all rows of `table` as one batch.
 * Replaces MaterializedExecutor.execute's rowPassesFilters +
 * computePartialAgg + finalizePartialAgg (src/client.ts:1023-1054). */
int qm_query_run(qm_ctx *ctx, const qm_table *table, const qm_query *query,
                 qm_result **out);

/* ---- streaming aggregation (AggregateOperator drop-in) ------------------ */
/* Begin an aggregation whose input arrives batch by batch, as
 * AggregateOperator.next drains upstream.nextColumnar
 * (src/operators.ts:1656-1681).  Filters in `query` are fused into the
 * aggregation kernel (the scan-time filter of src/operators.ts:439-547 plus
 * FilterOperator, src/operators.ts:1406-1496). */
int qm_agg_begin(qm_ctx *ctx, const qm_query *query, qm_agg **out);
/* Feed one batch: n_rows rows of n_cols columns (host or device).  If
 * `selection` is non-NULL it lists n_selected ascending row indices that are
 * alive (ColumnarBatch.selection, src/operators.ts:57-64); only those rows
 * are filtered and aggregated.  Row order across pushes is the batch order
 * the reference merges partials in. */
int qm_agg_push(qm_agg *agg, int64_t n_rows, int32_t n_cols,
                const qm_column *cols, const uint32_t *selection,
                int64_t n_selected);
/* Finalize into a result (src/partial-agg.ts:306-352). */
int qm_agg_finish(qm_agg *agg, qm_result **out);
int qm_agg_destroy(qm_agg *agg);

/* Push every row of a registered table as one batch (its columns are read
 * in place and its cached column statistics are used).  Same semantics as
 * qm_agg_push of those columns without a selection. */
int qm_agg_push_table(qm_agg *agg, const qm_table *table);

/* Partial group states across shards (multi-GPU).  The reference fans a
 * query out to fragment DOs and merges their partial aggregates
 * (src/query-do.ts:1747-1887, mergePartialAggs src/partial-agg.ts:277-304);
 * here each GPU streams its shard through its own qm_agg, exports the
 * occupied group slots as partial rows in device memory, and one GPU merges
 * the others' rows into its aggregation before qm_agg_finish.
 *
 * A partial row is *row_words 64-bit words: the group's key word, its
 * special flag (0; 1 key equal to the empty-slot sentinel; 2 NULL key) and
 * the aggregation's accumulator words.  Shards of one query over one schema
 * produce the same layout.  row_offset = the shard's first global row: FIRST
 * (first-seen order) moves by it.  With dst null only *n_groups and
 * *row_words are returned.  dst / src are device memory of this context's
 * GPU (copy other GPUs' rows in first: NCCL all-gather, peer copy). */
int qm_agg_partial_export(qm_agg *agg, int64_t row_offset, uint64_t *dst, int64_t capacity_rows,
                          int64_t *n_groups, int32_t *row_words);
/* rows_end: one past the last global row the partial covers (bounds the
 * first-seen sort). */
int qm_agg_partial_merge(qm_agg *agg, const uint64_t *src, int64_t n_groups, int32_t row_words,
                         int64_t rows_end);

/* The layout of this aggregation's partial rows: words per row and the word
 * holding the group's first global row (-1 when the query keeps no
 * first-seen order).  A finished result's rows come in ascending order of
 * that word. */
int qm_agg_partial_layout(const qm_agg *agg, int32_t *row_words, int32_t *first_word);
/* A new, empty aggregation with src's plan and partial-row layout, taking
 * only qm_agg_partial_merge: the receiving side of a key-partitioned
 * exchange, where each rank merges and finalizes the groups of its key
 * range.  (The reference reduces every fragment's partial on one node,
 * src/query-do.ts:1896-1960, src/merge.ts:156-172; splitting the groups
 * across ranks is this library's own step.) */
int qm_agg_partial_begin(const qm_agg *src, qm_agg **out);
/* Split n_rows partial rows (device memory of this context's GPU) into
 * `parts` groups by the hash of their key word, so that every rank's rows
 * of one group go to the same rank of an all-to-all exchange: dst (device,
 * n_rows rows) receives part 0's rows, then part 1's, ...; part_rows (host,
 * `parts` entries) receives each part's row count.  Rows of a special key
 * (the empty-slot sentinel, NULL) go to part 0.  1 <= parts <= 4096.  No
 * counterpart in the reference. */
int qm_partial_partition(qm_ctx *ctx, const uint64_t *src, int64_t n_rows, int32_t row_words, int32_t parts,
                         uint64_t *dst, int64_t *part_rows);

/* ---- filter-only selection (FilterOperator / WASM filter drop-in) ------- */
/* Evaluate the filters of `query` (aggregates and group_by ignored) over one
 * batch — over the rows listed by `selection` (ascending, n_selected) when it
 * is non-NULL, FilterOperator narrowing a selection vector
 * (src/operators.ts:1425-1466) — and write the ascending indices of passing
 * rows into out_indices
 * (capacity max_out).  Replaces filterFloat64Buffer / filterInt64Buffer /
 * filterInt32Buffer / *Range / *NotRange + intersectIndices / unionIndices
 * (wasm/src/wasm/aggregates.zig:605-1066) as composed by applyAndFilters /
 * scanFilterIndices (src/operators.ts:439-547).  If more than max_out rows
 * pass, *out_count is the full count and QM_ERR_CAPACITY is returned. */
int qm_filter_select(qm_ctx *ctx, int64_t n_rows, int32_t n_cols,
                     const qm_column *cols, const qm_query *query,
                     const uint32_t *selection, int64_t n_selected,
                     uint32_t *out_indices, int64_t max_out,
                     int64_t *out_count);

/* ---- filter -> GROUP BY without allocating --------------------------------- */
/* Bytes of the fixed device scratch array behind qm_query_run_noalloc. */
#define QM_NOALLOC_SCRATCH_BYTES (32u << 20)

/* No counterpart in the reference (its WASM engine owns a bump allocator).
 * For callers that cannot allocate device memory — code running inside
 * another framework's memory arena or allocator, or where cudaMalloc is not
 * available to it — this runs the query of qm_query_run over device-resident
 * columns without any device or pinned allocation: the group table and
 * every temporary live in one static device array of
 * QM_NOALLOC_SCRATCH_BYTES, held by each device from the library's module
 * load on it (its first call under lazy module loading) until the process
 * exits.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it; make that first call before any
 * stream capture, and make no call on a device after a cudaDeviceReset of
 * it.  Every call shares and re-initialises the array, so calls that
 * overlap on the GPU race: serialise them.
 * Without column statistics, a GROUP BY over several columns is limited to
 * two non-NULL int32 columns (QM_ERR_UNSUPPORTED otherwise; qm_query_run
 * packs other integer keys by their value ranges).
 *   cols         device columns only (on_device = 1); a NULL bitmap must be
 *                4-byte aligned and readable as ceil(n_rows/32) 32-bit words
 *   max_groups   capacity of the outputs; queries whose groups (or whose
 *                scratch need) exceed it fail with QM_ERR_CAPACITY
 *   out_columns  one device buffer per result column (keys, then aggregates),
 *                max_groups rows of the column's dtype (QM_I128 = 16 bytes)
 *   out_null_words  NULL or, per column, NULL or a device buffer of
 *                ceil(max_groups/32) 32-bit words receiving bit set = NULL
 *   out_dtypes   NULL or a host array receiving each result column's dtype
 *   out_groups   receives the number of groups written
 * Groups come in hash-table order, not first-seen order. */
int qm_query_run_noalloc(qm_ctx *ctx, int64_t n_rows, int32_t n_cols, const qm_column *cols,
                         const qm_query *query, int64_t max_groups, void *const *out_columns,
                         uint32_t *const *out_null_words, int32_t *out_dtypes, int64_t *out_groups);

/* ---- batched launch ------------------------------------------------------- */
typedef struct qm_batch qm_batch;

/* Plan n independent filter -> GROUP BY queries, query i over table i, for
 * one batched run (the reference runs them as n separate executions, each a
 * full pipeline, src/client.ts:1003-1085).  The queries are cut into waves;
 * each wave — table init, scans, first-seen ordering, finalize — is captured
 * as a CUDA graph on the first qm_batch_run and replayed afterwards, and its
 * packed results cross to host memory while later waves run (see
 * qm_batch_set_mode for the two ways a wave scans).  At most 4096 queries. */
int qm_batch_create(qm_ctx *ctx, int32_t n, const qm_table *const *tables,
                    const qm_query *const *queries, qm_batch **out);
/* Run the batch; results[i] receives query i's result (destroy each). */
int qm_batch_run(qm_batch *batch, qm_result **results);
/* Launch-shape knobs chosen by the autotuner (querymode_b200/autotune.py):
 * tiles of 256 rows per work chunk, block-local table budget in KiB (0:
 * global tables only), resident blocks per SM (0: occupancy).  A negative
 * value keeps the current setting.  Re-captures the graph on the next run. */
int qm_batch_set_tuning(qm_batch *batch, int32_t chunk_tiles, int32_t local_kb,
                        int32_t blocks_per_sm);
/* How the batch scans: 1 (default) one scan launch per query, each
 * specialised for its plan (value-column count, key kind) with the
 * planner's block-local table, spread over parallel stream branches of the
 * graph, largest query first; 0 persistent kernels, one per query class
 * (dedupe flag, value-column count, key kind) on parallel branches, whose
 * blocks claim (query, chunk of tiles) work items from the class's counter
 * and load each query's plan into shared memory (the chunk / local-table
 * knobs of qm_batch_set_tuning apply to them). */
int qm_batch_set_mode(qm_batch *batch, int32_t mode);
/* Waves of a batched run (0: by batch size, up to 8): the queries are cut
 * into waves run back to back, each followed by the copy of its results to
 * the host, which overlaps the later waves.  Queries whose results are large
 * for the bytes they scan go first.  Re-captures the graph on the next run. */
int qm_batch_set_waves(qm_batch *batch, int32_t waves);
/* Device time of the last run, total rows and algorithmic bytes, chunks. */
int qm_batch_stats(const qm_batch *batch, double *device_ms, int64_t *rows,
                   int64_t *bytes, int32_t *chunks);
int qm_batch_destroy(qm_batch *batch);

/* ---- Parquet column chunks ------------------------------------------------
 * Build a table from uncompressed Parquet column chunks: dictionary pages,
 * data pages v1 or v2 with PLAIN values or RLE_DICTIONARY / RLE indices
 * (encodings 8 and 3, the ones the reference reads as dictionary indices),
 * definition levels for optional columns:
 * the bytes the reference's decodeParquetColumnChunk reads
 * (src/parquet-decode.ts:390-618), decoded into HBM with the same results —
 * rows per page, NULLs from definition level 0, the v1 level section
 * recognised as the reference recognises it.  The chunk is the bytes from
 * the chunk's first page header (ColumnMetaData.data_page_offset) for
 * total_compressed_size bytes; num_values is ColumnMetaData.num_values.
 * Other encodings (PLAIN_DICTIONARY among them, which the reference would
 * read as PLAIN) and compressed pages give QM_ERR_UNSUPPORTED.  Every column
 * must decode to the same row count. */
typedef struct {
  const char *name;
  int32_t dtype;         /* QM_I32 / QM_I64 / QM_F32 / QM_F64: INT32 / INT64 / FLOAT / DOUBLE */
  int32_t reserved;
  const uint8_t *chunk;  /* host memory */
  int64_t chunk_bytes;
  int64_t num_values;
} qm_parquet_column;

int qm_table_from_parquet(qm_ctx *ctx, int32_t n_cols, const qm_parquet_column *cols, qm_table **out);
/* ---- Scan pages (Lance and Parquet) ----------------------------------------
 * Build a table from the page buffers a scan fetches: per column its pages in
 * order, decoded and concatenated as the reference's decodeAllColumns
 * (src/decode.ts:201-229) does.  A page with `parquet` set (PageInfo.encoding
 * present) is a Parquet column chunk of row_count values, decoded as
 * qm_table_from_parquet decodes it.  Any other page is decoded as decodePage
 * (src/decode.ts:251-331): PLAIN little-endian values; when null_count > 0
 * and row_count > 0 the page starts with a validity bitmap of
 * ceil(row_count / 8) bytes (bit set = a value), followed by either the
 * non-NULL values packed (data_offset < 0) or, from byte data_offset, one
 * slot per row (Lance v2 nullable pages, PageInfo.dataOffsetInPage).  Short
 * pages yield what the reference's decode yields (fewer rows, or NULLs where
 * the values run out).  Every column must decode to the same row count.
 * Pages are staged through pinned host buffers: many small pages become a few
 * DMA copies. */
typedef struct {
  const uint8_t *buf;   /* host memory */
  int64_t bytes;
  int64_t row_count;    /* PageInfo.rowCount (0: as many values as the bytes hold) */
  int64_t null_count;   /* PageInfo.nullCount */
  int64_t data_offset;  /* PageInfo.dataOffsetInPage, -1 when absent */
  int32_t parquet;      /* 1: PageInfo.encoding present, buf is a Parquet column chunk */
  int32_t reserved;
} qm_page;

/* Value types of PLAIN pages narrower than the table's dtypes, widened on
 * the device as the reference's numbers hold them (decodePlainValues,
 * src/parquet-decode.ts:280-386): int8 / uint8 / int16 / uint16 into QM_I32
 * columns, uint32 into QM_F64 (a JS number, exact), float16 into QM_F32
 * (exact).  QM_PT_SAME: the pages hold the column's dtype. */
#define QM_PT_SAME 0
#define QM_PT_INT8 1
#define QM_PT_UINT8 2
#define QM_PT_INT16 3
#define QM_PT_UINT16 4
#define QM_PT_UINT32 5
#define QM_PT_FLOAT16 6

typedef struct {
  const char *name;
  int32_t dtype;        /* QM_I32 / QM_I64 / QM_F32 / QM_F64 */
  int32_t n_pages;
  const qm_page *pages;
  int32_t page_type;    /* QM_PT_*: the value type of its (non-Parquet) pages */
  int32_t reserved;
} qm_page_column;

int qm_table_from_pages(qm_ctx *ctx, int32_t n_cols, const qm_page_column *cols, qm_table **out);

/* Copy a table column back to the host: values (n_rows cells of its dtype,
 * 0 where NULL) and/or one byte per row, 1 = NULL.  No counterpart in the
 * reference (inspection and tests). */
int qm_table_read_column(const qm_table *table, int32_t column, void *values, uint8_t *null_bytes);

/* ---- serving loop -----------------------------------------------------------
 * Continuous batching of single requests over resident tables.  The reference
 * serves each query in its own durable object (src/query-do.ts fan-out, one
 * single-threaded engine per object, src/wasm-engine.ts:181-186); here a
 * server runs several lanes, each a worker thread with its own CUDA stream:
 * a free lane takes the requests queued at that moment as one batched launch
 * (qm_batch_*), so requests that arrive while other batches run start on the
 * next free lane and their device work overlaps the others'.  Each request
 * completes as soon as its own result has been copied back.  A request over
 * a table of more than max_batch_rows rows is heavy: it runs alone, and the
 * light-only lane keeps small requests moving past it.
 *
 * HBM budget admission: the server counts the device bytes of every table
 * it has been given (resident) plus the working memory (group table,
 * bitmaps, packed result) of every request on the GPU.  A lane admits
 * queued requests in arrival order while resident + working bytes of all
 * lanes stay within hbm_budget_bytes; the rest wait until memory frees up.
 * A request that cannot fit even alone completes with QM_ERR_OOM.
 *
 * The server drives the context it is created on from its worker thread:
 * register tables first, and make no other call on that context (or its
 * tables) until qm_server_destroy returns.  submit / cancel / wait / stats
 * may be called from any thread. */
typedef struct qm_server qm_server;

typedef struct {
  int64_t hbm_budget_bytes; /* resident tables + working memory, bytes     */
  int32_t max_batch;        /* requests per batched launch (1..4096)       */
  int32_t max_wait_us;      /* the oldest queued request waits at most this
                               long for others before a launch (0: none)   */
  int64_t max_batch_rows;   /* rows a batch may scan (0: no limit); a
                               request over a table of more rows is heavy:
                               it runs alone, never on the light lane       */
  int32_t lanes;            /* batches in flight at once, each on its own
                               stream (0: 4); with more than one, the last
                               lane takes light requests only               */
  int32_t max_batch_groups; /* a request the planner sizes at more groups
                               than this (e.g. a 16M-group aggregate) is
                               heavy too: it runs alone, never on the light
                               lane (0: no limit)                          */
} qm_server_config;

typedef struct {
  int64_t queued_us;  /* submit -> launch of its batch                     */
  int64_t run_us;     /* launch -> result in host memory                   */
  int64_t total_us;   /* submit -> result in host memory                   */
  int32_t batch_size; /* requests in its batch                             */
  int32_t plan_us;    /* its lane planning and laying out the batch (host,
                         part of queued_us)                               */
} qm_server_timing;

typedef struct {
  int64_t submitted, completed, failed, cancelled, refused, batches;
  int64_t resident_bytes;     /* device bytes of the tables seen           */
  int64_t peak_working_bytes; /* most working memory of batches in flight  */
  int64_t queued;             /* requests waiting now                      */
  int64_t peak_in_flight;     /* most requests on the GPU at once          */
  int64_t heavy;              /* requests run alone as heavy               */
  int64_t lanes;              /* lanes of the server                       */
} qm_server_counters;

/* Start the lanes.  At creation the server page-locks 256 MB of result
 * buffers per lane (kept in the context's pinned pool) and takes up to 2 GB
 * per lane (at most an eighth of hbm_budget_bytes) from the device's memory
 * pool and hands it back, so that serving does not stall on page-locking or
 * pool growth later; qm_ctx_trim returns the device memory. */
int qm_server_create(qm_ctx *ctx, const qm_server_config *cfg, qm_server **out);
/* Queue one request (the query is copied; the table must stay alive).
 * *ticket identifies it for cancel / wait.  Planning errors surface from
 * qm_server_wait with the request's own code and message. */
int qm_server_submit(qm_server *srv, const qm_table *table, const qm_query *query,
                     uint64_t *ticket);
/* Cancel a request that has not been launched yet: its wait returns
 * QM_ERR_CANCELLED.  QM_ERR_INVALID if it is unknown, running or done. */
int qm_server_cancel(qm_server *srv, uint64_t ticket);
/* Wait for a request (timeout_us < 0: no limit; QM_ERR_TIMEOUT when it runs
 * out, the request stays pending) and take its result (destroy it) and
 * timing (may be null).  Returns the request's status; a ticket is
 * consumed by the wait that returns anything but QM_ERR_TIMEOUT.  The
 * message of a failed request is copied to msg (msg_len bytes) if given. */
int qm_server_wait(qm_server *srv, uint64_t ticket, int64_t timeout_us, qm_result **out,
                   qm_server_timing *timing, char *msg, size_t msg_len);
int qm_server_stats(qm_server *srv, qm_server_counters *out);
/* Stop the worker after the batch in flight and free the server.  Requests
 * not yet taken by a wait are dropped with their results; no wait may be in
 * progress. */
int qm_server_destroy(qm_server *srv);

/* ---- results ------------------------------------------------------------- */
int qm_result_num_rows(const qm_result *res, int64_t *out);
int qm_result_num_columns(const qm_result *res, int32_t *out);
int qm_result_column(const qm_result *res, int32_t index,
                     qm_result_col *out);
int qm_result_stats(const qm_result *res, qm_stats *out);
/* Encode the result as a QMCB buffer (src/columnar.ts:523-613), owned by
 * the result.  QM_I128 sums are written as I64 when every value fits, else
 * QM_ERR_UNSUPPORTED. */
int qm_result_qmcb(const qm_result *res, const uint8_t **buf, size_t *len);
int qm_result_destroy(qm_result *res);

#ifdef __cplusplus
}
#endif

#endif /* QM_GPU_H */
