// qm_batch.h — device-side description of a batch of queries (qm_batch.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "qm_plan.h"

#define QM_BATCH_MAX 4096

// One query of a batch.
struct qm_bq {
  qm_scan_args a;                  // plan, group table, status; a.n = rows
  qm_outspec outs;                 // offsets into the packed buffer (set on the device)
  int64_t bm_word0, bm_words;      // its slice of the batch's first-row bitmap
  int32_t none, pad;               // no GROUP BY: exactly one output row
  int32_t width[QM_MAX_OUT];       // bytes per row of each output column
  int32_t nullable[QM_MAX_OUT];
  int64_t nullbyte_off[QM_MAX_OUT];
};

// Work unit: tiles [tile0, tile1) of query q.
struct qm_chunk {
  int32_t q;
  int32_t pad;
  int64_t tile0, tile1;
};

struct qm_batch_meta {
  int64_t total;        // packed bytes of all results
  int64_t null_total;
  int64_t groups[QM_BATCH_MAX];
  int64_t base[QM_BATCH_MAX];
  int64_t bytes[QM_BATCH_MAX];
};

// Everything one batched run touches on the device.
struct qm_batch_dev {
  int n;
  int sm_count;
  qm_bq *bq;
  int64_t *slot0;       // n: first global slot of each query
  int64_t total_slots;
  qm_chunk *chunks;
  int n_chunks;
  int *counter;
  qm_status *statuses;
  uint32_t *bitmap;
  int64_t bm_words;
  uint32_t *popc;
  uint64_t *ranks;
  void *scan_temp;
  size_t scan_temp_bytes;
  qm_batch_meta *meta;
  qm_batch_meta *meta_host;  // pinned
  size_t meta_bytes;
  unsigned char *packed;
  unsigned char *nullbytes;
  uint32_t *perm;       // total_slots: slot of each ranked output row
};

size_t qm_batch_smem_bytes(int local_bytes);
// Per-class persistent launches: a query's class (dedupe flag, value-column
// count, key kind, fixed-point sums) picks a specialised instantiation of
// the persistent kernel (0: the run-time-plan one).  A wave keeps one work
// counter per class (QM_BATCH_CLASS_SLOTS counters from dev.counter).
#define QM_BATCH_CLASS_SLOTS 16
#define QM_BATCH_CLASSES_N 9
int qm_batch_class_of(const qm_scan_args &a);
// attr_smem: the class kernel's dynamic shared-memory limit to set (0: keep
// it); smem: the launch's shared memory for the occupancy answer.
cudaError_t qm_batch_class_configure(int cls, size_t attr_smem, size_t smem, int *blocks_per_sm);
cudaError_t qm_batch_launch_class(int cls, const qm_bq *bq, const qm_chunk *chunks, int n_chunks, int *counter,
                                  int local_bytes, int blocks, size_t smem, cudaStream_t st);
// The phases of a batched run: clear statuses, counters, bitmaps and group
// tables; the persistent scans (qm_batch_launch_class, one per class) or one
// specialised scan launch per query; rank, lay out, emit and pack the results.
cudaError_t qm_batch_launch_init(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_launch_finalize(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_scan_temp_bytes(int64_t words, size_t *bytes);
