// qm_plan.h — the lowered query plan shared by the host planner and the
// kernels.  Plain-old-data only: it is passed by value as a kernel parameter
// (single query) or copied into device memory (batched queries).
//
// A query is lowered into
//   * predicate terms  — filters normalised so the kernel evaluates each as
//     one integer range test or one IEEE comparison (the JS coercions of
//     src/decode.ts:480-541 are folded into the bounds on the host);
//   * a group key      — one 64-bit word per row (src/types.ts:10-18 builds a
//     string; for numeric columns string equality is equality of this word);
//   * accumulators     — the per-group state words of PartialAggState
//     (src/partial-agg.ts:13-36) that the query's aggregates read.
#pragma once
#include <stdint.h>

#define QM_MAX_TERMS 16
#define QM_MAX_VCOLS 8
#define QM_MAX_ACCS 16
#define QM_MAX_WORDS 24
#define QM_MAX_OUT 24
#define QM_R 8
// Zone maps: per column min / max over zones of QM_ZONE_TILES tiles
// (65,536 rows); zones the predicate cannot match are not scanned.
#define QM_ZONE_TILES 256
#define QM_ZONE_ROWS (QM_ZONE_TILES * 256)                   // rows per lane per warp tile
#define QM_TILE_ROWS (QM_R * 32) // rows per warp tile

// ---- predicate terms -------------------------------------------------------
enum qm_term_kind : int32_t {
  QT_TRUE = 0,      // constant pass (still subject to the NULL rule)
  QT_FALSE = 1,     // constant fail
  QT_IRANGE = 2,    // integer column: lo <= v <= hi
  QT_INRANGE = 3,   // integer column: v < lo || v > hi
  QT_FCMP = 4,      // float column: v <op> f0 (IEEE, NaN compares false)
  QT_FBETWEEN = 5,  // float column: v >= f0 && v <= f1
  QT_FNBETWEEN = 6, // float column: v < f0 || v > f1
  QT_FBIG = 7,      // float column vs bigint: BigInt(trunc(v)) <op> lo
  QT_FRANGE = 10,   // float column: v in (f0 | [f0) .. (f1 | f1]): op bit 0 = f0
                    // inclusive, bit 1 = f1 inclusive (NaN fails)
  QT_ISNULL = 8,
  QT_NOTNULL = 9,
};

enum qm_cmp_op : int32_t { QC_EQ = 0, QC_NEQ, QC_LT, QC_LTE, QC_GT, QC_GTE };

struct qm_term {
  const void *data;
  const uint32_t *nulls; // QMCB null bitmap viewed as 32-bit words, or null
  int32_t dtype;         // QM_I32 / QM_I64 / QM_F32 / QM_F64
  int32_t kind;          // qm_term_kind
  int32_t op;            // qm_cmp_op for QT_FCMP / QT_FBIG
  int32_t null_pass;     // result for a NULL cell: 0 (JS), or the result of
                         // the test on 0 (WASM scan reads NULL as 0)
  int32_t sidx;          // staged column holding this term's cells, or -1
  int32_t pad;
  int64_t lo, hi;
  double f0, f1;
};

struct qm_pred {
  int32_t n_and;                   // terms [0, n_and) are ANDed
  int32_t n_groups;                // OR groups after the AND terms
  int32_t group_end[QM_MAX_TERMS]; // group g = terms [end[g-1], end[g])
  qm_term t[QM_MAX_TERMS];
};

// ---- group key --------------------------------------------------------------
enum qm_key_mode : int32_t {
  QK_NONE = 0,   // no GROUP BY: one group
  QK_DIRECT = 1, // slot = key - base, for a dense integer key range
  QK_HASH = 2,   // open addressing on the 64-bit key
};

#define QM_MAX_KEYS 4

// How the key columns form the 64-bit key word.
enum qm_key_pack : int32_t {
  QP_RAW = 0,     // one column: its value (float: normalised bits)
  QP_CONCAT = 1,  // two non-null int32 columns: (u32)a << 32 | (u32)b
  QP_DIGITS = 2,  // integer columns as mixed-radix digits: digit_i = v - kbase_i
                  // (+1 when nullable, 0 = NULL), key = sum digit_i * kmul_i
};

struct qm_keyspec {
  int32_t n_cols;   // 0 .. QM_MAX_KEYS
  int32_t mode;     // qm_key_mode
  int32_t pack;     // qm_key_pack
  int32_t pad;
  const void *data[QM_MAX_KEYS];
  const uint32_t *nulls[QM_MAX_KEYS];
  int32_t dtype[QM_MAX_KEYS];
  int32_t knullable[QM_MAX_KEYS];
  int64_t kbase[QM_MAX_KEYS];
  uint64_t kmul[QM_MAX_KEYS];
  uint64_t kradix[QM_MAX_KEYS];
  int64_t base;     // QK_DIRECT: smallest key word
};

// ---- accumulators ----------------------------------------------------------
enum qm_acc_kind : int32_t {
  QA_COUNT = 0,  // rows in the group (COUNT(*)), u64
  QA_FIRST = 1,  // smallest global row index, u64 (first-seen order)
  QA_NN = 2,     // non-NULL cells of a column, u64
  QA_ISUM = 3,   // exact integer sum, 2 words: lo u64, hi i64
  QA_FSUM = 4,   // compensated float sum, 2 words: hi f64, lo f64
  QA_IMIN = 5,   // i64
  QA_IMAX = 6,   // i64
  QA_FMIN = 7,   // order-preserving i64 image of a double (-0 as +0)
  QA_FMAX = 8,
  QA_FZERO = 9,  // min over zero cells of (row << 1 | sign bit), u64
  QA_FNF = 10,   // non-finite cells of a fixed-point float SUM (atomic OR):
                 // bit 0 NaN, bit 1 +Infinity, bit 2 -Infinity
};

struct qm_acc {
  int32_t kind;
  int32_t vcol;  // value column index, -1 for COUNT / FIRST
  int32_t word;  // first word of the accumulator within a slot (after key)
  int32_t wide;  // QA_ISUM over int64 cells (128-bit even block-locally)
  int32_t narrow;  // QA_ISUM over int32 cells of a table below 2^32 rows:
                   // the sum fits a signed 64-bit word everywhere (the high
                   // word stays 0 and is the low word's sign at finalize)
  int32_t pad;
};

// Per value column: which accumulators read it (VF_* bits) and where their
// words live, so a row updates its slot in straight-line code.
#define VF_NN 1     // non-NULL count word
#define VF_SUM 2    // QA_ISUM (integer column) or QA_FSUM (float column)
#define VF_MIN 4
#define VF_MAX 8
#define VF_ZERO 16  // QA_FZERO (float MIN / MAX)
#define VF_WIDE 32  // 128-bit integer sum even block-locally (int64 cells)
#define VF_NARROW 64  // signed 64-bit integer sum in the global table too
#define VF_FIXED 128  // float SUM as an exact 128-bit fixed-point integer
                      // (units of 2^fx_exp): integer adds, so the sum does not
                      // depend on the order of the rows (deterministic)

struct qm_vcol {
  const void *data;
  const uint32_t *nulls;
  int32_t dtype;
  int32_t flags;
  int32_t w_nn, w_sum, w_min, w_max, w_zero, pad;
  // float SUM by error-free splitting: 1.5 * 2^(e+k) where every finite
  // |x| < 2^e and a group has fewer than 2^(k-1) rows; x splits exactly into
  // xh = (x + split) - split, a multiple of ulp(split) whose sums are exact in
  // any order, and xl = x - xh.  0: compensate each add with TwoSum instead.
  double split;
  // VF_FIXED: a finite cell x becomes round(x / 2^fx_exp) as a 128-bit
  // integer in the two QA_FSUM words (lo u64, hi i64); |x| must stay below
  // fx_max (else the kernel reports QM_DEV_STALE: the column's statistics
  // are out of date); non-finite cells set bits of word w_nf.
  int32_t fx_exp;
  int32_t w_nf;
  double fx_max;
};

struct qm_aggspec {
  int32_t n_accs;
  int32_t n_words;   // accumulator words per slot (excluding the key word)
  int32_t n_vcols;
  int32_t acc_count; // index of QA_COUNT / QA_FIRST in accs
  int32_t acc_first;
  int32_t w_count;   // word of QA_COUNT
  int32_t w_first;   // word of QA_FIRST, or -1
  int32_t pad;
  qm_acc acc[QM_MAX_ACCS];
  qm_vcol vcol[QM_MAX_VCOLS];
  uint64_t init[QM_MAX_WORDS]; // initial value of each accumulator word
};

// ---- outputs ---------------------------------------------------------------
enum qm_out_kind : int32_t {
  QO_KEY = 0,       // group key column `src`
  QO_COUNT = 1,     // u64 word -> int64
  QO_SUM_F = 2,     // FSUM -> double (NULL when nn == 0)
  QO_AVG_F = 3,     // FSUM / nn
  QO_SUM_I2F = 4,   // ISUM -> double (int32 column: JS number)
  QO_AVG_I2F = 5,   // ISUM / nn (int32 column)
  QO_SUM_I128 = 6,  // ISUM -> 128-bit (int64 column: JS bigint)
  QO_AVG_BIG = 7,   // bigAvg (src/partial-agg.ts:38-44), int64 column
  QO_MIN_I = 8,     // IMIN -> i64 or i32
  QO_MAX_I = 9,
  QO_MIN_F = 10,    // FMIN (+FZERO for the sign of a zero) -> double
  QO_MAX_F = 11,
};

struct qm_out {
  int32_t kind;
  int32_t dtype;    // result dtype (QM_I32 / QM_I64 / QM_F64 / QM_I128)
  int32_t word;     // main accumulator word
  int32_t nn_word;  // count word deciding NULL (and the AVG divisor)
  int32_t zero_word;// QA_FZERO word for float MIN/MAX, else -1
  int32_t src;      // key column index for QO_KEY
  int32_t narrow;   // QO_SUM_I2F / QO_AVG_I2F over a narrow (64-bit) sum
  int32_t fixed;    // QO_SUM_F / QO_AVG_F over a fixed-point sum (VF_FIXED)
  int32_t fx_exp;   //   its unit's exponent
  int32_t nf_word;  //   its QA_FNF word
  int32_t pad;
  int64_t offset;   // byte offset of the column in the output buffer
  int64_t null_offset; // byte offset of its 32-bit-word null bitmap, or -1
};

struct qm_outspec {
  int32_t n_out;
  int32_t pad;
  qm_out o[QM_MAX_OUT];
};

// ---- one launch of the fused filter + aggregate kernel ----------------------
#define QM_EMPTY_KEY 0x8000000000000000ULL // free hash slot; a real key equal
                                           // to it lives in a reserved slot
struct qm_status {
  int32_t error;      // QM_DEV_* below, first writer wins
  int32_t pad;
  unsigned long long rows_selected;
  unsigned long long groups_inserted; // new keys claimed in the global table
};
#define QM_DEV_OK 0
#define QM_DEV_OVERFLOW 1  // hash probe limit hit: regrow and re-run
#define QM_DEV_RANGE 2     // direct-mapped key outside the planned range
#define QM_DEV_TIMEOUT 3   // a bounded wait on an asynchronous copy gave up
#define QM_DEV_STALE 4     // a fixed-point SUM cell beyond the planned range:
                           // the column changed since its statistics were taken

// Filter columns copied tile by tile into shared memory with bulk async
// copies (cp.async.bulk + mbarrier), double buffered per warp.
#define QM_MAX_STAGED 4
#define QM_STAGE_MAX_DEPTH 4
struct qm_staging {
  int32_t n;                       // staged columns (0: read filters from global)
  int32_t tile_bytes;              // bytes of one tile of all staged columns
  int32_t depth;                   // tile buffers per warp (2..QM_STAGE_MAX_DEPTH)
  int32_t pad;
  const void *data[QM_MAX_STAGED];
  int32_t elem[QM_MAX_STAGED];     // 4 or 8
  int32_t off[QM_MAX_STAGED];      // byte offset of the column inside a tile buffer
};

struct qm_scan_args {
  qm_pred pred;
  qm_keyspec key;
  qm_aggspec agg;
  int64_t n;             // elements: rows, or selection entries when sel != 0
  const uint32_t *sel;   // ascending alive row indices, or null
  int64_t row_offset;    // global index of row 0 (batch order across pushes)
  uint64_t *table;       // group table: slot s = words [s*stride, (s+1)*stride)
  int64_t n_slots;       // QK_HASH capacity (power of two) / QK_DIRECT size
  int32_t stride;        // 1 key word + agg.n_words
  int32_t log2cap;       // QK_HASH
  int32_t local_slots;   // block-local table slots (0: none)
  int32_t local_hash;    // block-local table is hashed (else direct-indexed)
  int32_t dedupe;        // warp-level pre-aggregation of equal keys
  int32_t vec_ok;          // every term column is 16-byte aligned: vector loads
  int32_t max_probe;     // bound on linear probing in the global table
  int32_t priv;          // direct block-local table copied per warp: its
                         // (deduplicated) updates need no atomics
  const uint32_t *zones; // zones (QM_ZONE_TILES tiles each) to scan, ascending, or null: every tile
  int64_t n_zone_tiles;  // zones: tiles covered (count of zones x QM_ZONE_TILES)
  qm_status *status;
  qm_staging stage;
};

// ---- partitioned aggregation --------------------------------------------------
// For group tables larger than a block's shared memory: a counting pass and
// a scatter pass write every survivor as a record into its key partition
// (direct keys: a window of 2^shift slots; hashed keys: the top `bits` bits
// of the key's hash; special keys and direct keys outside the table: the
// last partition, `parts`), then one block per partition aggregates its
// records in a shared-memory table and merges it into the group table once.
// A record is 2 + value-column words: the key word; row (bits 0-31), special
// flag (32-39), NULL bits of the cells (40-47); the value cells.
struct qm_part_spec {
  int32_t parts;       // partitions of ordinary keys (partition `parts` takes the rest)
  int32_t direct;      // 1: partition = slot >> shift; 0: partition = hash >> (64 - bits)
  int32_t shift;
  int32_t bits;
  int32_t rec_words;
  int32_t blocks;      // grid of the counting and scatter passes (the same in both)
  int32_t local_slots; // slots of a partition's shared-memory table
  int32_t pad;
  int64_t rec_cap;     // records the buffer holds (a survivor past it is an overflow)
  uint32_t *counts;    // [(parts + 1) x blocks] survivors per partition and block
  uint64_t *offsets;   // [(parts + 1) x blocks] first record of each partition and block
  uint64_t *bases;     // [parts + 2] first record of each partition; then the total
  uint64_t *records;
  int *counter;        // partitions claimed by the aggregating blocks
};

// ---- Parquet column chunk decode (PLAIN pages) --------------------------------
// A page of a column chunk after its header was parsed on the host.
struct qm_pq_page {
  int64_t row0;     // first row of the page in the column
  int64_t rows;     // rows the page yields
  int64_t val_off;  // byte offset of its PLAIN values in the chunk
  int64_t avail;    // PLAIN values present (value bytes / width)
  int32_t run0;     // its definition-level runs: [run0, run1); none: every row present
  int32_t run1;
  int32_t slotted;  // 1: one value slot per row (NULL rows too), value j = row - row0;
                    // 0: present rows' values packed, value j = rank among present rows
  int32_t dict;     // 1: value j is dictionary entry index[j] (RLE_DICTIONARY page)
  int64_t dict_off; // dict: the dictionary's PLAIN values in the chunk, and how many
  int64_t dict_n;
  int64_t data_end; // dict: end of the page's data (index bytes at or past it read as 0)
  int64_t n_idx;    // dict: indices the page's index stream yields (index j >= n_idx: 0)
  int32_t irun0;    // dict: its index runs [irun0, irun1) (row0 = first index number)
  int32_t irun1;
  int32_t bw;       // dict: index bit width (0: every index 0)
  int32_t reserved;
};
// A run of the RLE / bit-packed hybrid definition levels (bit width 1).
struct qm_pq_run {
  int64_t row0;      // first row it covers (column-wide)
  int64_t count;     // rows it covers
  int64_t byte_off;  // bit-packed: its first data byte in the chunk
  int32_t packed;    // 1 bit-packed, 0 RLE
  int32_t value;     // RLE: the repeated level; bit-packed: data bytes present
                     // (levels past them read as 0)
};
