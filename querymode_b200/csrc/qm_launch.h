// qm_launch.h — host-callable launchers of the kernels in qm_kernels.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "qm_plan.h"

#define QM_SCAN_THREADS 512
#define QM_HLL_P 12

// Scan kernels specialised for N = 0..QM_SPEC_NV_MAX value columns
// (qm_scan_nvN.cu): dynamic shared memory limit of each, and the launch of
// the one for (dedupe flag, key kind QM_KK_*).
#define QM_SPEC_NV_MAX 4
#define QM_DECL_SPEC(N)                                                                        \
  cudaError_t qm_scan_nv##N##_attr(int max_smem);                                           \
  cudaError_t qm_scan_nv##N##_launch(const qm_scan_args &a, int dd, int kk, int blocks, size_t smem, \
                                     cudaStream_t st);
QM_DECL_SPEC(0)
QM_DECL_SPEC(1)
QM_DECL_SPEC(2)
QM_DECL_SPEC(3)
QM_DECL_SPEC(4)
#undef QM_DECL_SPEC

size_t qm_scan_smem_bytes(int local_slots, int local_hash, int n_words, int stage_tile_bytes, int stage_depth,
                          int priv);
cudaError_t qm_scan_configure(size_t smem_bytes, bool staged, int *blocks_per_sm);
cudaError_t qm_launch_scan(const qm_scan_args &a, int blocks, size_t smem_bytes, cudaStream_t st);
cudaError_t qm_launch_init_table(uint64_t *t, int64_t n_slots_total, int stride, int hash_keys,
                                 const qm_aggspec &A, int sm_count, cudaStream_t st);
cudaError_t qm_launch_compact(const uint64_t *t, int64_t n_slots_total, int stride, int count_word,
                              int first_word, uint64_t *keys_out, uint32_t *slots_out,
                              unsigned long long *counter, int sm_count, cudaStream_t st);
cudaError_t qm_sort_pairs(void *temp, size_t *temp_bytes, const uint64_t *kin, uint64_t *kout,
                          const uint32_t *vin, uint32_t *vout, int64_t n, int end_bit, cudaStream_t st);
cudaError_t qm_launch_emit(const uint64_t *t, int stride, const uint32_t *slots, int64_t G,
                           const qm_keyspec &K, int64_t n_slots, const qm_outspec &O, unsigned char *out,
                           int sm_count, cudaStream_t st);
cudaError_t qm_launch_select_masks(const qm_pred &P, int64_t n, const uint32_t *sel, uint32_t *masks,
                                   uint32_t *counts, int sm_count, cudaStream_t st);
cudaError_t qm_exclusive_scan_u32(void *temp, size_t *temp_bytes, const uint32_t *in, uint64_t *out, int64_t n,
                                  cudaStream_t st);
cudaError_t qm_launch_select_write(int64_t n_tiles, const uint32_t *sel, const uint32_t *masks,
                                   const uint64_t *offsets, uint32_t *out, int64_t max_out, int sm_count,
                                   cudaStream_t st);
cudaError_t qm_launch_minmax(const void *p, int dtype, const uint32_t *nulls, int64_t n, long long *out,
                             int sm_count, cudaStream_t st);
cudaError_t qm_launch_export_partial(const uint64_t *t, int stride, const uint32_t *slots, int64_t G, int64_t n_slots,
                                     int key_mode, const qm_aggspec &A, int64_t row_offset, uint64_t *dst, int sm_count,
                                     cudaStream_t st);
cudaError_t qm_launch_merge_partial(const qm_scan_args &a, const uint64_t *src, int64_t n, int sm_count,
                                    cudaStream_t st);
// Partial rows by key-hash part: per-part counts, then the rows into their
// parts' regions (cursor: each part's first row, advanced by the scatter).
cudaError_t qm_launch_partition_count(const uint64_t *src, int64_t n, int rw, int parts, unsigned long long *counts,
                                      int sm_count, cudaStream_t st);
cudaError_t qm_launch_partition_scatter(const uint64_t *src, int64_t n, int rw, int parts, unsigned long long *cursor,
                                        uint64_t *dst, int sm_count, cudaStream_t st);
// First-seen ranking of the occupied slots through a row bitmap and its
// prefix popcount (ranks[words] = number of groups), then the emit by rank.
cudaError_t qm_launch_rank_first(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                 uint32_t *bitmap, int64_t words, uint32_t *counts, uint64_t *ranks, void *temp,
                                 size_t temp_bytes, int sm_count, cudaStream_t st);
cudaError_t qm_rank_temp_bytes(int64_t words, size_t *bytes);
cudaError_t qm_launch_emit_ranked(const uint64_t *t, int64_t n_slots_total, int stride, int count_word,
                                  int first_word, const uint32_t *bitmap, const uint64_t *ranks, int64_t words,
                                  const qm_keyspec &K, int64_t n_slots, const qm_outspec &O, unsigned char *out,
                                  int sm_count, cudaStream_t st);
// Ranked emit in output order by walking the first-row bitmap: tables whose
// key columns hold every row the bitmap indexes (a: table, key, slots).
// bounds / chunk: walk only words [bounds[chunk], bounds[chunk + 1]) (bounds
// from qm_launch_walk_bounds; null: every word).
cudaError_t qm_launch_emit_walk(const qm_scan_args &a, const uint32_t *bitmap, const uint64_t *ranks, int64_t words,
                                const qm_outspec &O, unsigned char *out, int sm_count, cudaStream_t st,
                                const int64_t *bounds = nullptr, int chunk = 0);
// Ranked emit in two ordered steps (slot numbers to their ranks in perm,
// n_slots_total entries; then rows in order, at most `rows` of them).
cudaError_t qm_launch_emit_perm(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                const uint32_t *bitmap, const uint64_t *ranks, int64_t words, uint32_t *perm,
                                int64_t rows, const qm_keyspec &K, int64_t n_slots, const qm_outspec &O,
                                unsigned char *out, int sm_count, cudaStream_t st);
// First-seen order of a table of at most QM_SMALL_RANK_SLOTS slots in one
// block (perm: slot of each output row; groups[0]: their count), then the
// rows emitted in that order (at most `rows`).
#define QM_SMALL_RANK_SLOTS 2048
cudaError_t qm_launch_rank_small(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                 uint32_t *perm, uint64_t *groups, cudaStream_t st);
cudaError_t qm_launch_emit_sorted(const uint64_t *t, int stride, const uint32_t *perm, const uint64_t *groups,
                                  int64_t rows, const qm_keyspec &K, int64_t n_slots, const qm_outspec &O,
                                  unsigned char *out, int sm_count, cudaStream_t st);
// Word bounds (chunks + 1 entries) of output chunks of `per` rows.
cudaError_t qm_launch_walk_bounds(const uint64_t *ranks, int64_t words, int64_t per, int chunks, int64_t *bounds,
                                  cudaStream_t st);
// Post-aggregate ORDER BY / LIMIT over emitted result rows (see qm_kernels.cu).
cudaError_t qm_launch_sort_keys(const unsigned char *data, const uint32_t *nulls, int dtype, int desc, int64_t G,
                                uint32_t *last, uint64_t *hi, uint64_t *lo, uint32_t *idx, int sm_count, cudaStream_t st);
cudaError_t qm_stable_sort_rows(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, bool wide, int64_t G,
                                uint32_t *idx, uint32_t *idx2, uint64_t *k1, uint64_t *k2, uint32_t *l1, uint32_t *l2,
                                void *temp, size_t *temp_bytes, int sm_count, cudaStream_t st);
cudaError_t qm_launch_topk(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, int64_t G, int64_t k,
                           uint32_t *heap, uint32_t *out, cudaStream_t st);
// rows idx[first + j] (or first + j when idx is null), j < n
cudaError_t qm_launch_gather_rows(const unsigned char *src, const qm_outspec &O, const qm_outspec &O2,
                                  const uint32_t *idx, int64_t first, int64_t n, unsigned char *dst, int sm_count,
                                  cudaStream_t st);
// Decode a column from Parquet PLAIN pages (chunk bytes on the device; pages
// and definition-level runs parsed on the host).  temp null: *temp_bytes
// receives the scan's scratch size.  nulls may be null (no page has levels
// and none is a dictionary page).  iruns: the dictionary pages' index runs,
// null when no page is a dictionary page.
cudaError_t qm_launch_pq_decode(const uint8_t *chunk, const qm_pq_page *pages, int n_pages, const qm_pq_run *runs,
                                int n_runs, const qm_pq_run *iruns, int width, int in_width, int conv, int64_t n_rows, uint32_t *present, uint32_t *counts,
                                uint64_t *ranks, void *temp, size_t *temp_bytes, unsigned char *out, uint32_t *nulls,
                                int sm_count, cudaStream_t st);
cudaError_t qm_launch_zone_stats(const void *p, int dtype, const uint32_t *nulls, int64_t n, int64_t *zmin,
                                 int64_t *zmax, int64_t *zcount, cudaStream_t st);
cudaError_t qm_launch_sample_pred(const qm_pred &P, int64_t n, int n_samples, unsigned long long *count,
                                  cudaStream_t st);
cudaError_t qm_launch_hll(const qm_keyspec &K, int64_t n, uint32_t *regs, int sm_count, cudaStream_t st);
cudaError_t qm_launch_rehash(const uint64_t *old_t, int64_t old_cap, int stride, int count_word, uint64_t *new_t,
                             int log2cap, qm_status *st, int sm_count, cudaStream_t stream);
cudaError_t qm_launch_check_selection(const uint32_t *sel, int64_t n_sel, int64_t n_rows, qm_status *st,
                                      int sm_count, cudaStream_t stream);
cudaError_t qm_launch_maxabs(const void *p, int dtype, const uint32_t *nulls, int64_t n, unsigned long long *out,
                             int sm_count, cudaStream_t st);

// Partitioned aggregation (qm_part.cu): the counting pass (pass 0) or the
// scatter pass (pass 1) over the plan's rows, the per-partition offsets, and
// the aggregation of each partition's records.
size_t qm_part_scan_smem(int parts);
int qm_part_scan_blocks(int sm_count, int parts);
cudaError_t qm_launch_part_scan(int pass, const qm_scan_args &a, const qm_part_spec &ps, cudaStream_t st);
cudaError_t qm_launch_part_offsets(const qm_part_spec &ps, cudaStream_t st);
size_t qm_part_agg_smem(int local_slots, int local_hash, int n_words);
cudaError_t qm_launch_part_agg(const qm_scan_args &a, const qm_part_spec &ps, int sm_count, cudaStream_t st);

// The library's exclusive scan: scratch bytes for n inputs, and ranks of a
// bitmap (ranks[i] = set bits in words before i, ranks[words] = all of them).
size_t qm_scan_temp_bytes_for(int64_t n);
cudaError_t qm_scan_popc_words(const uint32_t *bitmap, int64_t words, uint64_t *ranks, void *temp, size_t temp_bytes,
                               cudaStream_t st);
