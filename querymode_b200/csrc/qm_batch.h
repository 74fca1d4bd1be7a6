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
  int scan_blocks;
  size_t scan_smem;
  int local_bytes;
};

size_t qm_batch_smem_bytes(int local_bytes);
cudaError_t qm_batch_configure(size_t smem, int *blocks_per_sm);
// The three phases of a batched run: clear statuses, bitmaps and group
// tables; the persistent scan over every query's chunks (or, instead, one
// specialised scan launch per query issued by the host); rank, lay out,
// emit and pack the results.
cudaError_t qm_batch_launch_init(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_launch_persistent(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_launch_finalize(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_launch_all(const qm_batch_dev &d, cudaStream_t st);
cudaError_t qm_batch_scan_temp_bytes(int64_t words, size_t *bytes);
