// qm_kernels.cu — kernels of the filter -> GROUP BY path and their launchers.
//
//   qm_scan_kernel      fused filter + compaction + group-by aggregation
//   qm_init_table       fill the group table with empty keys / initial words
//   qm_compact_groups   list occupied slots with their first-seen row
//   qm_emit_groups      finalize each group's row (src/partial-agg.ts:306-352)
//   qm_select_masks /   filter-only selection vector (ascending row indices)
//   qm_select_write
//   qm_minmax_kernel    integer column min / max (planning statistics)
#include <cuda_fp16.h>
#include <cub/cub.cuh>

#include <climits>

#include <mutex>

#include "qm_scan.cuh"

namespace qm {

// ---- partial group states across shards (multi-GPU) --------------------------
// A partial row is [key word, special (0, 1 = sentinel-valued key, 2 = NULL
// key), accumulator words].  Export moves FIRST / FZERO by the shard's first
// global row, so merged tables keep the global first-seen order.
__global__ void qm_export_partial(const uint64_t *t, int stride, const uint32_t *slots, int64_t G, int64_t n_slots,
                                  int key_mode, const __grid_constant__ qm_aggspec A, int64_t row_offset,
                                  uint64_t *dst) {
  const int rw = stride + 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = slots ? (int64_t)slots[i] : 0;
    const uint64_t *w = t + s * stride;
    uint64_t *o = dst + i * rw;
    int special = 0;
    if (key_mode == QK_HASH) special = s == n_slots ? 1 : (s == n_slots + 1 ? 2 : 0);
    o[0] = key_mode == QK_NONE ? 0 : (special == 1 ? QM_EMPTY_KEY : (special == 2 ? 0 : w[0]));
    o[1] = (uint64_t)special;
    for (int k = 0; k < A.n_words; ++k) o[2 + k] = w[1 + k];
    for (int k = 0; k < A.n_accs; ++k) {
      const qm_acc ac = A.acc[k];
      uint64_t &v = o[2 + ac.word];
      if (ac.kind == QA_FIRST && v != ~0ULL) v += (uint64_t)row_offset;
      if (ac.kind == QA_FZERO && v != ~0ULL) v += (uint64_t)row_offset << 1;
    }
  }
}

// Key-partitioned exchange of partial rows: the part of a row is the hash of
// its key word modulo the part count (rows of a special key go to part 0),
// so every rank's rows of one group meet on one rank.
__device__ __forceinline__ int partial_part(const uint64_t *row, int parts) {
  return row[1] != 0 ? 0 : (int)(fmix64(row[0] ^ 0x9e3779b97f4a7c15ULL) % (uint64_t)parts);
}

__global__ void qm_partition_count(const uint64_t *src, int64_t n, int rw, int parts, unsigned long long *counts) {
  extern __shared__ unsigned long long hist[];
  for (int p = threadIdx.x; p < parts; p += blockDim.x) hist[p] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&hist[partial_part(src + i * rw, parts)], 1ULL);
  __syncthreads();
  for (int p = threadIdx.x; p < parts; p += blockDim.x)
    if (hist[p]) atomicAdd(&counts[p], hist[p]);
}

// Rows to their part's region: lanes of a warp bound for the same part take
// consecutive places with one atomic (the order inside a part is free: the
// merge does not depend on it).
__global__ void qm_partition_scatter(const uint64_t *src, int64_t n, int rw, int parts,
                                     unsigned long long *cursor, uint64_t *dst) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const int64_t i = base + threadIdx.x;
    const bool live = i < n;
    const unsigned act = __ballot_sync(QM_FULL, live);
    if (!live) continue;
    const int p = partial_part(src + i * rw, parts);
    const unsigned peers = __match_any_sync(act, p);
    const int leader = __ffs(peers) - 1;
    unsigned long long at = 0;
    if (lane == leader) at = atomicAdd(&cursor[p], (unsigned long long)__popc(peers));
    at = __shfl_sync(peers, at, leader) + __popc(peers & ((1u << lane) - 1));
    const uint64_t *r = src + i * rw;
    uint64_t *o = dst + (int64_t)at * rw;
    for (int k = 0; k < rw; ++k) o[k] = r[k];
  }
}

// Fold partial rows into the group table (slots found / claimed as in the
// scan); integer sums are 128-bit, float sums compensated (TwoSum).
__global__ void qm_merge_partial(const __grid_constant__ qm_scan_args a, const uint64_t *src, int64_t n) {
  const qm_aggspec &A = a.agg;
  const int rw = a.stride + 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t *row = src + i * rw;
    const int64_t gs = global_slot(a, row[0], (int)row[1]);
    if (gs < 0) continue;
    uint64_t *gp = a.table + gs * a.stride + 1;
    const uint64_t *v = row + 2;
    for (int k = 0; k < A.n_accs; ++k) {
      const qm_acc ac = A.acc[k];
      const uint64_t v0 = v[ac.word];
      uint64_t *g0 = gp + ac.word, *g1 = gp + ac.word + 1;
      switch (ac.kind) {
        case QA_COUNT:
        case QA_NN:
          if (v0) atomicAdd(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
          break;
        case QA_FIRST:
        case QA_FZERO:
          if (v0 != ~0ULL) atomicMin(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
          break;
        case QA_ISUM:
          if (ac.narrow) {
            if (v0) atomicAdd(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
          } else if (v0 || v[ac.word + 1]) {
            add128(g0, g1, v0, (int64_t)v[ac.word + 1]);
          }
          break;
        case QA_FSUM:
          if (A.vcol[ac.vcol].flags & VF_FIXED) {
            if (v0 || v[ac.word + 1]) add128(g0, g1, v0, (int64_t)v[ac.word + 1]);
          } else {
            fsum_add(g0, g1, __longlong_as_double((long long)v0), __longlong_as_double((long long)v[ac.word + 1]));
          }
          break;
        case QA_FNF:
          if (v0) atomicOr(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
          break;
        case QA_IMIN:
        case QA_FMIN:
          if ((int64_t)v0 != (int64_t)A.init[ac.word]) atomicMin(reinterpret_cast<long long *>(g0), (long long)v0);
          break;
        case QA_IMAX:
        case QA_FMAX:
          if ((int64_t)v0 != (int64_t)A.init[ac.word]) atomicMax(reinterpret_cast<long long *>(g0), (long long)v0);
          break;
      }
    }
  }
}

// Filter pass count over a strided sample of rows (row i*n/n_samples):
// planning sizes a filtered query's group table by min(distinct keys,
// selected rows), and the sample bounds the selected rows.
__global__ void qm_sample_pred(const __grid_constant__ qm_pred P, int64_t n, int n_samples,
                               unsigned long long *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = i < n_samples ? (int64_t)i * n / n_samples : 0;
  uint32_t m = i < n_samples ? 1u : 0u;
  auto rowf = [&](int) { return r; };
  m = eval_pred(P, rowf, m);
  const unsigned b = __ballot_sync(QM_FULL, m & 1u);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, (unsigned long long)__popc(b));
}

__global__ void qm_init_table(uint64_t *t, int64_t n_slots_total, int stride, int hash_keys,
                              const __grid_constant__ qm_aggspec A) {
  const int64_t n = n_slots_total * stride;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int w = (int)(i % stride);
    t[i] = w == 0 ? (hash_keys ? QM_EMPTY_KEY : 0ULL) : A.init[w - 1];
  }
}

// Occupied slots (COUNT word > 0) with their sort key: the first-seen row
// (or the slot itself when no order is needed).
__global__ void qm_compact_groups(const uint64_t *t, int64_t n_slots_total, int stride, int count_word,
                                  int first_word, uint64_t *keys_out, uint32_t *slots_out,
                                  unsigned long long *counter) {
  const int lane = threadIdx.x & 31;
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t s0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); s0 < n_slots_total; s0 += step) {
    const int64_t s = s0 + lane;
    const bool occ = s < n_slots_total && t[s * stride + 1 + count_word] > 0;
    const unsigned b = __ballot_sync(QM_FULL, occ);
    if (!b) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, (unsigned long long)__popc(b));
    base = __shfl_sync(QM_FULL, base, 0);
    if (occ) {
      const unsigned long long pos = base + __popc(b & lanemask_lt());
      keys_out[pos] = first_word >= 0 ? t[s * stride + 1 + first_word] : (uint64_t)s;
      slots_out[pos] = (uint32_t)s;
    }
  }
}

// Move the occupied hash slots of a table into a larger one (keys are
// unique, so each new slot has one writer and the words are plain copies).
__global__ void qm_rehash(const uint64_t *old_t, int64_t old_cap, int stride, int count_word, uint64_t *new_t,
                          int log2cap, qm_status *st) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < old_cap; s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t *src = old_t + s * stride;
    if (src[1 + count_word] == 0) continue;
    const int64_t ns = global_find(new_t, stride, log2cap, src[0], 1 << 12, st);
    if (ns < 0) {
      set_error(st, QM_DEV_OVERFLOW);
      continue;
    }
    uint64_t *dst = new_t + ns * stride;
    for (int w = 1; w < stride; ++w) dst[w] = src[w];
  }
}

__global__ void qm_emit_groups(const uint64_t *t, int stride, const uint32_t *slots, int64_t G,
                               const __grid_constant__ qm_keyspec K, int64_t n_slots,
                               const __grid_constant__ qm_outspec O, unsigned char *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < G;
       i += (int64_t)gridDim.x * blockDim.x)
    emit_group<false>(t, stride, slots ? slots[i] : (uint64_t)i, i, K, n_slots, O, out, nullptr, nullptr);
}

// First-seen ranking without a sort: bit `first row` of every occupied slot
// in a row bitmap (each row belongs to one group, so bits are distinct);
// the prefix popcount of the bitmap then gives each group's output row.
// (a FIRST row outside the bitmap's `words` words is left unmarked: it can
// only come from a table the status reports as failed, whose result is
// discarded)
__global__ void qm_mark_first(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                              uint32_t *bitmap, int64_t words) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_slots_total;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t *w = t + s * stride + 1;
    if (w[count_word] == 0) continue;
    const uint64_t f = w[first_word];
    if ((f >> 5) >= (uint64_t)words) continue;
    atomicOr(bitmap + (f >> 5), 1u << (f & 31));
  }
}


__global__ void qm_emit_ranked(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                               const uint32_t *bitmap, const uint64_t *ranks, int64_t words,
                               const __grid_constant__ qm_keyspec K, int64_t n_slots,
                               const __grid_constant__ qm_outspec O, unsigned char *out) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_slots_total;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t *w = t + s * stride + 1;
    if (w[count_word] == 0) continue;
    const uint64_t f = w[first_word];
    if ((f >> 5) >= (uint64_t)words) continue;  // not marked (see qm_mark_first)
    const int64_t i = (int64_t)ranks[f >> 5] + __popc(bitmap[f >> 5] & ((1u << (f & 31)) - 1u));
    emit_group<false>(t, stride, (uint64_t)s, i, K, n_slots, O, out, nullptr, nullptr);
  }
}

// The same output in two ordered steps, for large results of any table:
// every occupied slot writes its number at its rank (4-byte stores into an
// array that stays in L2), then each output row reads its slot, so the output
// cells are written in runs instead of one scattered cell per column.
__global__ void qm_rank_slots(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                              const uint32_t *bitmap, const uint64_t *ranks, int64_t words, uint32_t *perm) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_slots_total;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t *w = t + s * stride + 1;
    if (w[count_word] == 0) continue;
    const uint64_t f = w[first_word];
    if ((f >> 5) >= (uint64_t)words) continue;  // not marked (see qm_mark_first)
    const int64_t i = (int64_t)ranks[f >> 5] + __popc(bitmap[f >> 5] & ((1u << (f & 31)) - 1u));
    if (i < n_slots_total) perm[i] = (uint32_t)s;
  }
}

// First-seen order of a small table (at most QM_SMALL_RANK_SLOTS slots) in
// one block: the occupied slots are collected with their first rows into
// shared memory and sorted by first row (bitonic; first rows are distinct),
// their slot numbers written in that order to perm and their count to
// groups[0] (one launch where the bitmap ranking takes five).
__global__ void __launch_bounds__(1024) qm_rank_small(const uint64_t *t, int64_t n_slots_total, int stride,
                                                      int count_word, int first_word, uint32_t *perm,
                                                      uint64_t *groups) {
  __shared__ uint64_t fr[QM_SMALL_RANK_SLOTS];
  __shared__ uint32_t sl[QM_SMALL_RANK_SLOTS];
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int64_t s = threadIdx.x; s < n_slots_total && s < QM_SMALL_RANK_SLOTS; s += blockDim.x) {
    const uint64_t *w = t + s * stride + 1;
    if (w[count_word] == 0) continue;
    const int i = atomicAdd(&cnt, 1);
    fr[i] = w[first_word];
    sl[i] = (uint32_t)s;
  }
  __syncthreads();
  const int n = cnt;
  int P = 1;
  while (P < n) P <<= 1;
  for (int i = n + (int)threadIdx.x; i < P; i += blockDim.x) {
    fr[i] = ~0ULL;
    sl[i] = 0;
  }
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool up = (i & k) == 0;
          if ((fr[i] > fr[ixj]) == up) {
            const uint64_t f = fr[i];
            fr[i] = fr[ixj];
            fr[ixj] = f;
            const uint32_t v = sl[i];
            sl[i] = sl[ixj];
            sl[ixj] = v;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sl[i];
  if (threadIdx.x == 0) groups[0] = (uint64_t)n;
}

// rows: the layout's capacity (output rows past it are not written).
__global__ void qm_emit_perm(const uint64_t *t, int stride, const uint32_t *perm, const uint64_t *ranks,
                             int64_t words, int64_t rows, const __grid_constant__ qm_keyspec K, int64_t n_slots,
                             const __grid_constant__ qm_outspec O, unsigned char *out) {
  const int64_t G = min((int64_t)ranks[words], rows);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x)
    emit_group<false>(t, stride, (uint64_t)perm[i], i, K, n_slots, O, out, nullptr, nullptr);
}

// The same output in output order, for a table whose key columns still hold
// every row the first-row bitmap indexes: output row i is the group whose
// first row is the i-th set bit, and that row's key finds the group's slot
// (a: the table, its key and slot layout).  Consecutive threads take consecutive bitmap words, so the
// output columns are written in runs (the slot-order emit scatters every
// 8-byte cell to its rank, and a result of millions of groups then costs a
// partial-sector write per cell).
// bounds (optional): this launch walks words [bounds[chunk], bounds[chunk + 1]).
__global__ void qm_emit_walk(const __grid_constant__ qm_scan_args a, const uint32_t *bitmap, const uint64_t *ranks,
                             int64_t words, const __grid_constant__ qm_outspec O, unsigned char *out,
                             const int64_t *bounds, int chunk) {
  const int64_t w0 = bounds ? bounds[chunk] : 0, w1 = bounds ? bounds[chunk + 1] : words;
  for (int64_t w = w0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < w1; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t b = bitmap[w];
    if (b == 0) continue;
    int64_t i = (int64_t)ranks[w];
    for (; b; b &= b - 1, ++i) {
      const int64_t r = w * 32 + (__ffs(b) - 1);
      int special;
      const uint64_t key = row_key<QM_KK_ANY>(a.key, r, special);
      const int64_t s = find_slot(a, key, special);
      if (s < 0) continue;  // not a group of this table (a failed run's bitmap)
      emit_group<false>(a.table, a.stride, (uint64_t)s, i, a.key, a.n_slots, O, out, nullptr, nullptr);
    }
  }
}

// Bitmap word bounds of output chunks of `per` rows: bounds[c] = the first
// word whose rank is at least c * per (lower bound over ranks[0..words]),
// bounds[chunks] = words.  A word's later bits may fall into the next
// chunk's rows; no word of a later chunk writes rows of an earlier one.
__global__ void qm_walk_bounds(const uint64_t *ranks, int64_t words, int64_t per, int chunks, int64_t *bounds) {
  const int c = threadIdx.x;
  if (c > chunks) return;
  if (c == chunks) {
    bounds[c] = words;
    return;
  }
  const uint64_t target = (uint64_t)c * (uint64_t)per;
  int64_t lo = 0, hi = words;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (ranks[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  bounds[c] = lo;
}

// ---- Parquet PLAIN pages -> a column ----------------------------------------
// (src/parquet-decode.ts:390-618: decodeParquetColumnChunk's PLAIN path, and
// decodePage, src/decode.ts:251-331)
__device__ __forceinline__ int pq_find_page(const qm_pq_page *pages, int n, int64_t r) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pages[mid].row0 <= r) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The contiguous range of 32-row words this warp decodes: pages and runs
// are then found once and followed forward.
__device__ __forceinline__ void pq_warp_range(int64_t words, int64_t &w0, int64_t &w1) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t per = (words + warps - 1) / warps;
  w0 = min(words, wid * per);
  w1 = min(words, w0 + per);
}

// The page a lane is in, held in registers and followed forward.
struct PqCur {
  int p;
  int64_t row0, next0, val_off, avail;
  int32_t run0, run1, slotted, dict;
  __device__ __forceinline__ void load(const qm_pq_page *pages, int n_pages, int q) {
    p = q;
    const qm_pq_page &pg = pages[q];
    row0 = pg.row0;
    val_off = pg.val_off;
    avail = pg.avail;
    run0 = pg.run0;
    run1 = pg.run1;
    slotted = pg.slotted;
    dict = pg.dict;
    next0 = q + 1 < n_pages ? pages[q + 1].row0 : INT64_MAX;
  }
  __device__ __forceinline__ bool advance(const qm_pq_page *pages, int n_pages, int64_t r) {
    if (r < next0) return false;
    int q = p;
    while (q + 1 < n_pages && pages[q + 1].row0 <= r) ++q;
    load(pages, n_pages, q);
    return true;
  }
};

// Presence bits, one lane per row: definition level 1 (a value) or 0 (NULL)
// from the page's level runs; pages without runs are all present, and so are
// rows past the levels decoded (the reference's `undefined !== 0`).
__global__ void __launch_bounds__(256) qm_pq_present(const uint8_t *chunk, const qm_pq_page *pages, int n_pages,
                                                     const qm_pq_run *runs, int64_t n_rows, uint32_t *present) {
  const int lane = threadIdx.x & 31;
  const int64_t words = (n_rows + 31) / 32;
  int64_t w0, w1;
  pq_warp_range(words, w0, w1);
  if (w0 >= w1) return;
  PqCur c;
  c.load(pages, n_pages, pq_find_page(pages, n_pages, min(w0 * 32 + lane, n_rows - 1)));
  int ri = -1;
  int64_t run_row0 = 0, run_end = -1, run_next = INT64_MAX, run_off = 0;
  int32_t run_packed = 0, run_value = 0;
  for (int64_t w = w0; w < w1; ++w) {
    const int64_t r = w * 32 + lane;
    bool on = false;
    if (r < n_rows) {
      if (c.advance(pages, n_pages, r)) ri = -1;
      if (c.run0 >= c.run1) {
        on = true;
      } else {
        if (ri < 0 || r >= run_next) {
          if (ri < 0) {  // the run holding r: binary search within the page
            int lo = c.run0, hi = c.run1 - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (runs[mid].row0 <= r) lo = mid;
              else hi = mid - 1;
            }
            ri = lo;
          }
          while (ri + 1 < c.run1 && runs[ri + 1].row0 <= r) ++ri;
          const qm_pq_run &run = runs[ri];
          run_row0 = run.row0;
          run_end = run.row0 + run.count;
          run_off = run.byte_off;
          run_packed = run.packed;
          run_value = run.value;
          run_next = ri + 1 < c.run1 ? runs[ri + 1].row0 : INT64_MAX;
        }
        const int64_t k = r - run_row0;
        if (k < 0 || r >= run_end) on = true;
        else if (run_packed) on = (k >> 3) < run_value && ((chunk[run_off + (k >> 3)] >> (k & 7)) & 1);
        else on = run_value & 1;
      }
    }
    const uint32_t bits = __ballot_sync(QM_FULL, on);
    if (lane == 0) present[w] = bits;
  }
}

// Dictionary page: the address of the entry value j of the page maps to
// (index j of its RLE / bit-packed index stream; index bytes at or past the
// page's data end read as 0, indices past those decoded are 0), or null
// where the index is outside the dictionary (NULL, as the reference's
// `idx < dictionary.length ? dictionary[idx] : null`).
__device__ __forceinline__ const uint8_t *pq_dict_entry(const uint8_t *chunk, const qm_pq_page &pg,
                                                       const qm_pq_run *iruns, int64_t j, int width) {
  uint64_t idx = 0;
  if (j < pg.n_idx) {
    int lo = pg.irun0, hi = pg.irun1 - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (iruns[mid].row0 <= j) lo = mid;
      else hi = mid - 1;
    }
    const qm_pq_run &run = iruns[lo];
    if (!run.packed) {
      idx = (uint32_t)run.value;
    } else {
      const int64_t bit = (j - run.row0) * pg.bw;
      const int64_t b0 = run.byte_off + (bit >> 3);
      uint64_t word = 0;
#pragma unroll
      for (int i = 0; i < 5; ++i)
        if (b0 + i < pg.data_end) word |= (uint64_t)chunk[b0 + i] << (8 * i);
      idx = (word >> (bit & 7)) & (pg.bw >= 32 ? 0xffffffffull : ((1ull << pg.bw) - 1));
    }
  }
  if (idx >= (uint64_t)pg.dict_n) return nullptr;
  return chunk + pg.dict_off + (int64_t)idx * width;
}

// Values into rows, one lane per row, QM_PQ_UNROLL words per step with their
// loads issued together (stores coalesced).  A present row r of page p
// takes that page's value j: in a packed page j = rank(r) - rank(row0), in
// a slotted page (or any page of a column without levels: present == null)
// j = r - row0.  j past the values present gives NULL (as the reference's
// decoded[dPtr++] / values[vi++] running out does).
// A page value of in_width bytes widened to the column's cell (conv: the
// QM_PT_* page type; int8 / uint8 / int16 / uint16 to int32, uint32 to a
// double, float16 to a float, each exact).
__device__ __forceinline__ uint64_t pq_widen(uint64_t v, int conv) {
  switch (conv) {
    case 1: return (uint64_t)(uint32_t)(int32_t)(int8_t)(v & 0xff);
    case 2: return v & 0xff;
    case 3: return (uint64_t)(uint32_t)(int32_t)(int16_t)(v & 0xffff);
    case 4: return v & 0xffff;
    case 5: return (uint64_t)__double_as_longlong((double)(uint32_t)v);
    case 6: return (uint64_t)__float_as_uint(__half2float(__ushort_as_half((unsigned short)(v & 0xffff))));
    default: return v;
  }
}

// DICT: the column has dictionary pages; WIDE: page values narrower than the
// column's (in_width bytes, widened by conv).  Separate instantiations, so
// the PLAIN one keeps its registers (five blocks per SM).
#define QM_PQ_UNROLL 4
template <bool DICT, bool WIDE>
__global__ void __launch_bounds__(256, (DICT || WIDE) ? 4 : 5)
    qm_pq_scatter(const uint8_t *chunk, const qm_pq_page *pages, int n_pages, const qm_pq_run *iruns, int width,
                  int in_width, int conv, int64_t n_rows, const uint32_t *present, const uint64_t *ranks,
                  unsigned char *out, uint32_t *nulls) {
  const int lane = threadIdx.x & 31;
  const int64_t words = (n_rows + 31) / 32;
  int64_t w0, w1;
  pq_warp_range(words, w0, w1);
  if (w0 >= w1) return;
  PqCur c;
  c.load(pages, n_pages, pq_find_page(pages, n_pages, min(w0 * 32 + lane, n_rows - 1)));
  int rank_p = -1;  // page whose first-row rank is in rank_f
  int64_t rank_f = 0;
  for (int64_t w = w0; w < w1; w += QM_PQ_UNROLL) {
    const uint8_t *src[QM_PQ_UNROLL];
    bool live[QM_PQ_UNROLL];
#pragma unroll
    for (int u = 0; u < QM_PQ_UNROLL; ++u) {
      const int64_t r = (w + u) * 32 + lane;
      live[u] = false;
      src[u] = nullptr;
      if (w + u < w1 && r < n_rows) {
        c.advance(pages, n_pages, r);
        const uint32_t pw = present ? present[w + u] : QM_FULL;
        if ((pw >> lane) & 1) {
          int64_t j;
          if (c.slotted || !present) {
            j = r - c.row0;
          } else {
            if (rank_p != c.p) {
              const int64_t f = c.row0;
              rank_f = (int64_t)ranks[f >> 5] + __popc(present[f >> 5] & ((1u << (f & 31)) - 1u));
              rank_p = c.p;
            }
            j = (int64_t)ranks[w + u] + __popc(pw & ((1u << lane) - 1u)) - rank_f;
          }
          if (DICT && c.dict) {
            src[u] = pq_dict_entry(chunk, pages[c.p], iruns, j, width);
            live[u] = src[u] != nullptr;
          } else if (j < c.avail) {
            live[u] = true;
            src[u] = chunk + c.val_off + j * (WIDE ? in_width : width);
          }
        }
      }
    }
    uint64_t v[QM_PQ_UNROLL];
#pragma unroll
    for (int u = 0; u < QM_PQ_UNROLL; ++u) {
      v[u] = 0;
      if (live[u]) {
        const uint8_t *s = src[u];
        if (WIDE) {
          if (((uintptr_t)s & (in_width - 1)) == 0) {
            v[u] = in_width == 4 ? *(const uint32_t *)s : in_width == 2 ? *(const uint16_t *)s : *s;
          } else {
            for (int i = in_width - 1; i >= 0; --i) v[u] = (v[u] << 8) | s[i];
          }
          v[u] = pq_widen(v[u], conv);
        } else if (((uintptr_t)s & (width - 1)) == 0) {
          v[u] = width == 8 ? *(const uint64_t *)s : *(const uint32_t *)s;
        } else {
          for (int i = width - 1; i >= 0; --i) v[u] = (v[u] << 8) | s[i];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < QM_PQ_UNROLL; ++u) {
      const int64_t r = (w + u) * 32 + lane;
      if (w + u < w1) {
        if (r < n_rows) {
          if (width == 8) ((uint64_t *)out)[r] = v[u];
          else ((uint32_t *)out)[r] = (uint32_t)v[u];
        }
        const uint32_t nb = __ballot_sync(QM_FULL, !live[u] && r < n_rows);
        if (nulls && lane == 0) nulls[w + u] = nb;
      }
    }
  }
}

// ---- zone maps -----------------------------------------------------------------
// Per zone of QM_ZONE_ROWS rows: min and max of the non-NULL cells (integer
// columns as int64; float columns as doubles, NaN excluded) and how many
// such cells there are.  One block per zone.
__global__ void qm_zone_stats(const void *p, int dtype, const uint32_t *nulls, int64_t n, int64_t *zmin,
                              int64_t *zmax, int64_t *zcount) {
  const int64_t z = blockIdx.x;
  const int64_t r0 = z * QM_ZONE_ROWS, r1 = min(n, r0 + (int64_t)QM_ZONE_ROWS);
  const bool isf = dtype == QM_F64 || dtype == QM_F32;
  long long mn = LLONG_MAX, mx = LLONG_MIN, cnt = 0;
  double fmn = INFINITY, fmx = -INFINITY;
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    if (cell_null(nulls, r)) continue;
    if (isf) {
      const double d = ld_flt(p, dtype, r);
      if (isnan(d)) continue;
      fmn = fmin(fmn, d);
      fmx = fmax(fmx, d);
    } else {
      const long long v = ld_int(p, dtype, r);
      mn = min(mn, v);
      mx = max(mx, v);
    }
    ++cnt;
  }
  for (int o = 16; o; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(QM_FULL, mn, o));
    mx = max(mx, __shfl_xor_sync(QM_FULL, mx, o));
    fmn = fmin(fmn, __shfl_xor_sync(QM_FULL, fmn, o));
    fmx = fmax(fmx, __shfl_xor_sync(QM_FULL, fmx, o));
    cnt += __shfl_xor_sync(QM_FULL, cnt, o);
  }
  __shared__ long long smn[32], smx[32], scnt[32];
  __shared__ double sfmn[32], sfmx[32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smn[w] = mn;
    smx[w] = mx;
    scnt[w] = cnt;
    sfmn[w] = fmn;
    sfmx[w] = fmx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
      mn = min(mn, smn[i]);
      mx = max(mx, smx[i]);
      cnt += scnt[i];
      fmn = fmin(fmn, sfmn[i]);
      fmx = fmax(fmx, sfmx[i]);
    }
    if (isf) {
      zmin[z] = __double_as_longlong(fmn);
      zmax[z] = __double_as_longlong(fmx);
    } else {
      zmin[z] = mn;
      zmax[z] = mx;
    }
    zcount[z] = cnt;
  }
}

// ---- post-aggregate ORDER BY / LIMIT on the emitted result rows ------------
// A row's sort value under rowComparator (src/types.ts:26-38): NULL and NaN
// are "last" in either direction; other values compare as JS numbers /
// bigints (exactly: int32 / int64 / 128-bit integers, IEEE doubles with -0
// equal to 0).  key = an unsigned 128-bit image ordered like the value,
// bit-inverted for descending order, so ascending key order is output order.
__device__ __forceinline__ void sort_key(const unsigned char *data, const uint32_t *nulls, int dtype, int desc,
                                         int64_t i, uint32_t &last, uint64_t &hi, uint64_t &lo) {
  last = (nulls && ((nulls[i >> 5] >> (i & 31)) & 1u)) ? 1u : 0u;
  hi = 0;
  lo = 0;
  if (!last) {
    switch (dtype) {
      case QM_I32: lo = (uint64_t)(int64_t)reinterpret_cast<const int32_t *>(data)[i] ^ (1ULL << 63); break;
      case QM_I64: lo = (uint64_t)reinterpret_cast<const int64_t *>(data)[i] ^ (1ULL << 63); break;
      case QM_I128:
        lo = reinterpret_cast<const uint64_t *>(data)[2 * i];
        hi = reinterpret_cast<const uint64_t *>(data)[2 * i + 1] ^ (1ULL << 63);
        break;
      default: {
        double d = reinterpret_cast<const double *>(data)[i];
        if (isnan(d)) {
          last = 1u;
        } else {
          if (d == 0.0) d = 0.0;
          lo = (uint64_t)f2ord(d) ^ (1ULL << 63);
        }
      }
    }
  }
  if (last) {
    hi = 0;
    lo = 0;
  } else if (desc) {
    hi = ~hi;
    lo = ~lo;
  }
}

__global__ void qm_sort_keys(const unsigned char *data, const uint32_t *nulls, int dtype, int desc, int64_t G,
                             uint32_t *last, uint64_t *hi, uint64_t *lo, uint32_t *idx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t l;
    uint64_t h, w;
    sort_key(data, nulls, dtype, desc, i, l, h, w);
    last[i] = l;
    hi[i] = h;
    lo[i] = w;
    idx[i] = (uint32_t)i;
  }
}

// x[i] = src[idx[i]] (the next key of an LSD radix sort, in the order so far)
__global__ void qm_gather_u64(const uint64_t *src, const uint32_t *idx, int64_t n, uint64_t *x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = src[idx[i]];
}
__global__ void qm_gather_u32(const uint32_t *src, const uint32_t *idx, int64_t n, uint32_t *x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = src[idx[i]];
}

// TopKOperator (src/operators.ts:1716-1841) over result rows 0..G-1 in
// order, exactly: a max-heap of k row indices under the reference's cmp
// (worse rows toward the root), a row replacing the root only when strictly
// better, extraction by repeated root removal, reversed.  The heap itself is
// sequential (one thread, as in the reference); rows are screened against
// the root in parallel first: the root only improves, so a row that does not
// beat the root at the start of its chunk cannot enter later in the chunk.
__device__ __forceinline__ int topk_cmp(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, uint32_t a,
                                        uint32_t b) {
  const uint32_t la = last[a], lb = last[b];
  if (la && lb) return 0;
  if (la) return 1;
  if (lb) return -1;
  if (hi[a] != hi[b]) return hi[a] < hi[b] ? -1 : 1;
  if (lo[a] != lo[b]) return lo[a] < lo[b] ? -1 : 1;
  return 0;
}

__device__ __forceinline__ bool topk_better(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, uint32_t r,
                                            uint32_t root) {
  if (last[r]) return false;
  if (last[root]) return true;
  if (hi[r] != hi[root]) return hi[r] < hi[root];
  return lo[r] < lo[root];
}

__device__ void topk_sift_down(uint32_t *h, int64_t n, int64_t i, const uint32_t *last, const uint64_t *hi,
                               const uint64_t *lo) {
  for (;;) {
    int64_t t = i;
    const int64_t l = 2 * i + 1, r = 2 * i + 2;
    if (l < n && topk_cmp(last, hi, lo, h[l], h[t]) > 0) t = l;
    if (r < n && topk_cmp(last, hi, lo, h[r], h[t]) > 0) t = r;
    if (t == i) break;
    const uint32_t x = h[i];
    h[i] = h[t];
    h[t] = x;
    i = t;
  }
}

#define QM_TOPK_THREADS 1024
__global__ void __launch_bounds__(QM_TOPK_THREADS)
    qm_topk_heap(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, int64_t G, int64_t k, uint32_t *heap,
                 uint32_t *out) {
  __shared__ uint32_t cand[QM_TOPK_THREADS];
  __shared__ int n_cand;
  __shared__ long long hlen;
  if (threadIdx.x == 0) hlen = 0;
  __syncthreads();
  for (int64_t base = 0; base < G; base += QM_TOPK_THREADS) {
    const int64_t i = base + threadIdx.x;
    const long long len = hlen;
    bool c = i < G && k > 0;
    if (c && len >= k) c = topk_better(last, hi, lo, (uint32_t)i, heap[0]);
    if (threadIdx.x == 0) n_cand = 0;
    __syncthreads();
    // keep the candidates in row order: warp ballots, warps in turn
    const unsigned bal = __ballot_sync(QM_FULL, c);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int wcount[QM_TOPK_THREADS / 32];
    if (lane == 0) wcount[warp] = __popc(bal);
    __syncthreads();
    if (c) {
      int off = 0;
      for (int w = 0; w < warp; ++w) off += wcount[w];
      cand[off + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)i;
    }
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < QM_TOPK_THREADS / 32; ++w) tot += wcount[w];
      n_cand = tot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long n = hlen;
      for (int j = 0; j < n_cand; ++j) {
        const uint32_t r = cand[j];
        if (n < k) {  // push + sift up
          int64_t x = n++;
          heap[x] = r;
          while (x > 0) {
            const int64_t p = (x - 1) >> 1;
            if (topk_cmp(last, hi, lo, heap[x], heap[p]) > 0) {
              const uint32_t y = heap[x];
              heap[x] = heap[p];
              heap[p] = y;
              x = p;
            } else {
              break;
            }
          }
        } else if (n > 0 && topk_better(last, hi, lo, r, heap[0])) {
          heap[0] = r;
          topk_sift_down(heap, n, 0, last, hi, lo);
        }
      }
      hlen = n;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    // extraction: root first (the worst kept), then reversed
    long long n = hlen;
    const long long total = n;
    for (long long e = 0; n > 0; ++e) {
      out[total - 1 - e] = heap[0];
      heap[0] = heap[n - 1];
      --n;
      if (n > 0) topk_sift_down(heap, n, 0, last, hi, lo);
    }
  }
}

// Copy the selected result rows (idx[0..n)) of every output column, with
// their NULL bits, into a second result buffer laid out for n rows.
__global__ void qm_gather_rows(const unsigned char *src, const __grid_constant__ qm_outspec O,
                               const __grid_constant__ qm_outspec O2, const uint32_t *idx, int64_t first, int64_t n,
                               unsigned char *dst) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx ? (int64_t)idx[first + j] : first + j;
    for (int k = 0; k < O.n_out; ++k) {
      const int w = O.o[k].dtype == QM_I128 ? 16 : (O.o[k].dtype == QM_I32 ? 4 : 8);
      const unsigned char *s = src + O.o[k].offset + i * w;
      unsigned char *d = dst + O2.o[k].offset + j * w;
      for (int b = 0; b < w; b += 4) *reinterpret_cast<uint32_t *>(d + b) = *reinterpret_cast<const uint32_t *>(s + b);
      if (O.o[k].null_offset >= 0) {
        const uint32_t *sn = reinterpret_cast<const uint32_t *>(src + O.o[k].null_offset);
        if ((sn[i >> 5] >> (i & 31)) & 1u)
          atomicOr(reinterpret_cast<uint32_t *>(dst + O2.o[k].null_offset) + (j >> 5), 1u << (j & 31));
      }
    }
  }
}

// Filter-only pass 1: per warp tile, the 32-bit survivor masks and counts.
template <bool SEL>
__global__ void __launch_bounds__(QM_SCAN_THREADS)
    qm_select_masks(const __grid_constant__ qm_pred P, int64_t n, const uint32_t *sel, uint32_t *masks,
                    uint32_t *counts) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const int64_t n_tiles = (n + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  for (int64_t tile = (int64_t)blockIdx.x * warps + (threadIdx.x >> 5); tile < n_tiles;
       tile += (int64_t)gridDim.x * warps) {
    const int64_t e0 = tile * QM_TILE_ROWS;
    int64_t rowv[QM_R];
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < QM_R; ++j) {
      int64_t e = e0 + j * 32 + lane;
      bool in = e < n;
      m |= (uint32_t)in << j;
      rowv[j] = SEL ? (in ? (int64_t)__ldg(sel + e) : 0) : e;
    }
    auto rowf = [&](int j) { return rowv[j]; };
    m = eval_pred(P, rowf, m);
    uint32_t tot = 0;
#pragma unroll
    for (int j = 0; j < QM_R; ++j) {
      uint32_t b = __ballot_sync(QM_FULL, (m >> j) & 1);
      if (lane == j) masks[tile * QM_R + j] = b;
      tot += __popc(b);
    }
    if (lane == 0) counts[tile] = tot;
  }
}

// Filter-only pass 2: ascending row indices at each tile's exclusive offset.
__global__ void qm_select_write(int64_t n_tiles, const uint32_t *sel, const uint32_t *masks,
                                const uint64_t *offsets, uint32_t *out, int64_t max_out) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const uint32_t lt = lanemask_lt();
  for (int64_t tile = (int64_t)blockIdx.x * warps + (threadIdx.x >> 5); tile < n_tiles;
       tile += (int64_t)gridDim.x * warps) {
    uint64_t pos = offsets[tile];
    const int64_t e0 = tile * QM_TILE_ROWS;
    for (int j = 0; j < QM_R; ++j) {
      const uint32_t b = masks[tile * QM_R + j];
      if ((b >> lane) & 1) {
        const uint64_t p = pos + __popc(b & lt);
        const int64_t e = e0 + j * 32 + lane;
        if ((int64_t)p < max_out) out[p] = sel ? __ldg(sel + e) : (uint32_t)e;
      }
      pos += __popc(b);
    }
  }
}

// min / max of a (possibly nullable) integer column.
__global__ void qm_minmax_kernel(const void *p, int dtype, const uint32_t *nulls, int64_t n,
                                 long long *out) {
  long long mn = LLONG_MAX, mx = LLONG_MIN;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (cell_null(nulls, i)) continue;
    long long v = dtype == QM_I32 ? (long long)__ldg((const int *)p + i) : __ldg((const long long *)p + i);
    mn = min(mn, v);
    mx = max(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(QM_FULL, mn, o));
    mx = max(mx, __shfl_xor_sync(QM_FULL, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, mn);
    atomicMax(out + 1, mx);
  }
}

// A selection vector must list strictly ascending row indices below n_rows.
__global__ void qm_check_selection(const uint32_t *sel, int64_t n_sel, int64_t n_rows, qm_status *st) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_sel; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = sel[i];
    if ((int64_t)v >= n_rows || (i > 0 && sel[i - 1] >= v)) set_error(st, QM_DEV_RANGE);
  }
}

// HyperLogLog registers (2^QM_HLL_P) of the group keys: the planner's
// distinct-count estimate that sizes hash tables.
__global__ void qm_hll_kernel(const __grid_constant__ qm_keyspec K, int64_t n, uint32_t *regs) {
  __shared__ uint32_t r[1 << QM_HLL_P];
  for (int i = threadIdx.x; i < (1 << QM_HLL_P); i += blockDim.x) r[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int special;
    uint64_t key = row_key(K, i, special);
    if (special == 2) key = 0x6e756c6c6e756c6cULL;
    const uint64_t h = fmix64(key ^ 0x9e3779b97f4a7c15ULL);
    const uint32_t idx = (uint32_t)(h >> (64 - QM_HLL_P));
    const uint64_t w = h << QM_HLL_P;
    const uint32_t rank = w ? (uint32_t)__clzll((long long)w) + 1 : (uint32_t)(65 - QM_HLL_P);
    atomicMax(&r[idx], rank);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << QM_HLL_P); i += blockDim.x)
    if (r[i]) atomicMax(&regs[i], r[i]);
}

// max |x| over the finite non-NULL cells of a float column (as the bits of a
// non-negative double, which order like unsigned integers).
__global__ void qm_maxabs_kernel(const void *p, int dtype, const uint32_t *nulls, int64_t n,
                                 unsigned long long *out) {
  unsigned long long mx = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (cell_null(nulls, i)) continue;
    const double v = dtype == QM_F32 ? (double)__ldg((const float *)p + i) : __ldg((const double *)p + i);
    if (!isfinite(v)) continue;
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v));
    mx = b > mx ? b : mx;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(QM_FULL, mx, o);
    mx = x > mx ? x : mx;
  }
  if ((threadIdx.x & 31) == 0 && mx) atomicMax(out, mx);
}

__global__ void qm_minmax_init(long long *out) {
  out[0] = LLONG_MAX;
  out[1] = LLONG_MIN;
}

}  // namespace qm

// ---------------------------------------------------------------- launchers
using namespace qm;

// ---- exclusive scan (u32 or popcounts of u32 words -> u64) -------------------
// Three phases without waits between blocks: every block sums its tile of
// SCAN_TILE inputs; one block turns the tile sums into tile offsets; every
// block scans its tile again (thread sums, warp shuffles, one shared-memory
// pass over the warps) and adds its tile's offset.  out[n] receives the
// total.  POPC: the inputs are bitmap words and count their set bits.
#define QM_SCAN_BLOCK 256
#define QM_SCAN_PER 8
#define QM_SCAN_TILE (QM_SCAN_BLOCK * QM_SCAN_PER)

template <bool POPC>
__device__ __forceinline__ uint64_t scan_in(const uint32_t *in, int64_t i, int64_t n) {
  if (i >= n) return 0;
  const uint32_t x = in[i];
  return POPC ? (uint64_t)__popc(x) : (uint64_t)x;
}

// A thread's QM_SCAN_PER inputs; VEC: two 16-byte loads when all 8 are in range
// (the caller checked that `in` is 16-byte aligned; base is a multiple of 8).
template <bool POPC, bool VEC>
__device__ __forceinline__ void scan_load8(const uint32_t *in, int64_t base, int64_t n, uint64_t (&v)[QM_SCAN_PER]) {
  if (VEC && base + QM_SCAN_PER <= n) {
    const uint4 a = reinterpret_cast<const uint4 *>(in + base)[0];
    const uint4 b = reinterpret_cast<const uint4 *>(in + base)[1];
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int k = 0; k < QM_SCAN_PER; ++k) v[k] = POPC ? (uint64_t)__popc(w[k]) : (uint64_t)w[k];
  } else {
#pragma unroll
    for (int k = 0; k < QM_SCAN_PER; ++k) v[k] = scan_in<POPC>(in, base + k, n);
  }
}

template <bool POPC, bool VEC>
__global__ void __launch_bounds__(QM_SCAN_BLOCK) qm_scan_tile_sums(const uint32_t *in, int64_t n, uint64_t *sums) {
  __shared__ uint64_t wsum[QM_SCAN_BLOCK / 32];
  const int64_t base = (int64_t)blockIdx.x * QM_SCAN_TILE + (int64_t)threadIdx.x * QM_SCAN_PER;
  uint64_t v[QM_SCAN_PER];
  scan_load8<POPC, VEC>(in, base, n, v);
  uint64_t t = 0;
#pragma unroll
  for (int k = 0; k < QM_SCAN_PER; ++k) t += v[k];
#pragma unroll
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(QM_FULL, t, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t b = 0;
    for (int w = 0; w < QM_SCAN_BLOCK / 32; ++w) b += wsum[w];
    sums[blockIdx.x] = b;
  }
}

// one block: tile sums -> exclusive tile offsets (in place), total at
// sums[tiles].  Each thread sums a run of tiles; the runs' sums are scanned
// by warp shuffles (lanes, then the warps' totals in warp 0).
__global__ void __launch_bounds__(1024) qm_scan_tile_offsets(uint64_t *sums, int64_t tiles) {
  __shared__ uint64_t wtot[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t per = (tiles + blockDim.x - 1) / blockDim.x;
  const int64_t b0 = (int64_t)threadIdx.x * per;
  uint64_t t = 0;
  for (int64_t i = 0; i < per; ++i)
    if (b0 + i < tiles) t += sums[b0 + i];
  uint64_t x = t;  // inclusive scan of the runs across the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(QM_FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wtot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = (int)(blockDim.x >> 5);
    const uint64_t w = lane < nw ? wtot[lane] : 0;
    uint64_t z = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(QM_FULL, z, o);
      if (lane >= o) z += y;
    }
    if (lane < nw) wtot[lane] = z - w;  // exclusive
    if (lane == 31) sums[tiles] = z;
  }
  __syncthreads();
  uint64_t acc = wtot[warp] + x - t;  // exclusive offset of this thread's run
  __syncthreads();  // every run's sums read before any is overwritten
  for (int64_t i = 0; i < per; ++i)
    if (b0 + i < tiles) {
      const uint64_t v = sums[b0 + i];
      sums[b0 + i] = acc;
      acc += v;
    }
}

// VEC: 16-byte loads and stores for full runs of 8 (the caller checked that
// `in` and `out` are 16-byte aligned).
template <bool POPC, bool VEC>
__global__ void __launch_bounds__(QM_SCAN_BLOCK)
    qm_scan_tiles(const uint32_t *in, int64_t n, const uint64_t *offsets, uint64_t *out, int write_total) {
  __shared__ uint64_t wsum[QM_SCAN_BLOCK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * QM_SCAN_TILE + (int64_t)threadIdx.x * QM_SCAN_PER;
  uint64_t v[QM_SCAN_PER];
  scan_load8<POPC, VEC>(in, base, n, v);
  uint64_t t = 0;
#pragma unroll
  for (int k = 0; k < QM_SCAN_PER; ++k) t += v[k];
  uint64_t x = t;  // inclusive scan of thread sums across the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(QM_FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t acc = 0;
    for (int w = 0; w < QM_SCAN_BLOCK / 32; ++w) {
      const uint64_t y = wsum[w];
      wsum[w] = acc;
      acc += y;
    }
  }
  __syncthreads();
  uint64_t run = offsets[blockIdx.x] + wsum[warp] + x - t;  // exclusive offset of this thread's first input
  if (VEC && base + QM_SCAN_PER <= n) {
    uint64_t r[QM_SCAN_PER];
#pragma unroll
    for (int k = 0; k < QM_SCAN_PER; ++k) {
      r[k] = run;
      run += v[k];
    }
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + base);
#pragma unroll
    for (int k = 0; k < QM_SCAN_PER / 2; ++k) o[k] = make_ulonglong2(r[2 * k], r[2 * k + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < QM_SCAN_PER; ++k) {
      if (base + k < n) out[base + k] = run;
      run += v[k];
    }
  }
  if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = offsets[gridDim.x];
}

// Scratch bytes of qm_scan_u64 over n inputs.
size_t qm_scan_temp_bytes_for(int64_t n) {
  return (size_t)(((n + QM_SCAN_TILE - 1) / QM_SCAN_TILE) + 2) * sizeof(uint64_t);
}

// out[i] = sum of inputs before i, i < n; with write_total also out[n] = the
// total (out then holds n + 1 entries).
template <bool POPC>
cudaError_t qm_scan_u64(const uint32_t *in, int64_t n, uint64_t *out, void *temp, size_t temp_bytes,
                        cudaStream_t st, bool write_total = true) {
  const int64_t tiles = std::max<int64_t>((n + QM_SCAN_TILE - 1) / QM_SCAN_TILE, 1);
  if (temp_bytes < qm_scan_temp_bytes_for(n)) return cudaErrorInvalidValue;
  uint64_t *sums = static_cast<uint64_t *>(temp);
  const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
  if (vec) qm_scan_tile_sums<POPC, true><<<(unsigned)tiles, QM_SCAN_BLOCK, 0, st>>>(in, n, sums);
  else qm_scan_tile_sums<POPC, false><<<(unsigned)tiles, QM_SCAN_BLOCK, 0, st>>>(in, n, sums);
  qm_scan_tile_offsets<<<1, 1024, 0, st>>>(sums, tiles);
  if (vec) qm_scan_tiles<POPC, true><<<(unsigned)tiles, QM_SCAN_BLOCK, 0, st>>>(in, n, sums, out, write_total ? 1 : 0);
  else qm_scan_tiles<POPC, false><<<(unsigned)tiles, QM_SCAN_BLOCK, 0, st>>>(in, n, sums, out, write_total ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t qm_scan_popc_words(const uint32_t *bitmap, int64_t words, uint64_t *ranks, void *temp, size_t temp_bytes,
                               cudaStream_t st) {
  return qm_scan_u64<true>(bitmap, words, ranks, temp, temp_bytes, st);
}


size_t qm_scan_smem_bytes(int local_slots, int local_hash, int n_words, int stage_tile_bytes, int stage_depth,
                          int priv) {
  return make_smem_layout(local_slots, local_hash, n_words, QM_SCAN_THREADS / 32, stage_tile_bytes, stage_depth, priv)
      .bytes;
}

namespace {
constexpr int QM_SCAN_SMEM_MAX = 227 * 1024 - 1024;  // dynamic, beside the kernel's static words

// Raise every scan kernel's dynamic shared memory limit to the maximum, once
// per device (launches then pass their actual size).
cudaError_t scan_attrs_once() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && done[dev]) return cudaSuccess;
#define QM_SMEM_ATTR(K) \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, QM_SCAN_SMEM_MAX);
  QM_SMEM_ATTR((qm_scan_kernel<false, true, 0, QM_NV_ANY, QM_KK_ANY>));
  QM_SMEM_ATTR((qm_scan_kernel<false, true, 1, QM_NV_ANY, QM_KK_ANY>));
  QM_SMEM_ATTR((qm_scan_kernel<false, false, 0, QM_NV_ANY, QM_KK_ANY>));
  QM_SMEM_ATTR((qm_scan_kernel<false, false, 1, QM_NV_ANY, QM_KK_ANY>));
  QM_SMEM_ATTR((qm_scan_kernel<true, false, 0, QM_NV_ANY, QM_KK_ANY>));
  QM_SMEM_ATTR((qm_scan_kernel<true, false, 1, QM_NV_ANY, QM_KK_ANY>));
#undef QM_SMEM_ATTR
  if (e == cudaSuccess) e = qm_scan_nv0_attr(QM_SCAN_SMEM_MAX);
  if (e == cudaSuccess) e = qm_scan_nv1_attr(QM_SCAN_SMEM_MAX);
  if (e == cudaSuccess) e = qm_scan_nv2_attr(QM_SCAN_SMEM_MAX);
  if (e == cudaSuccess) e = qm_scan_nv3_attr(QM_SCAN_SMEM_MAX);
  if (e == cudaSuccess) e = qm_scan_nv4_attr(QM_SCAN_SMEM_MAX);
  if (e == cudaSuccess && dev < 64) done[dev] = true;
  return e;
}

// Key kind of a plan for the specialised kernels (QM_KK_*).
int key_kind(const qm_keyspec &K) {
  if (K.n_cols == 0) return QM_KK_NONE;
  if (K.n_cols == 1 && K.pack == QP_RAW && K.nulls[0] == nullptr) {
    if (K.dtype[0] == QM_I64) return QM_KK_I64;
    if (K.dtype[0] == QM_I32) return QM_KK_I32;
  }
  return QM_KK_ANY;
}
}  // namespace

cudaError_t qm_scan_configure(size_t smem_bytes, bool staged, int *blocks_per_sm) {
  if (smem_bytes > (size_t)QM_SCAN_SMEM_MAX) return cudaErrorInvalidValue;
  cudaError_t e = scan_attrs_once();
  if (e != cudaSuccess) return e;
  if (staged)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        blocks_per_sm, qm_scan_kernel<false, true, 0, QM_NV_ANY, QM_KK_ANY>, QM_SCAN_THREADS, smem_bytes);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks_per_sm, qm_scan_kernel<false, false, 0, QM_NV_ANY, QM_KK_ANY>, QM_SCAN_THREADS, smem_bytes);
}

cudaError_t qm_launch_scan(const qm_scan_args &a, int blocks, size_t smem_bytes, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  cudaError_t e = scan_attrs_once();
  if (e != cudaSuccess) return e;
  const int dd = a.dedupe != 0 ? 1 : 0;
  // fixed-point (deterministic) sums run in the run-time-plan kernels only
  bool fixed = false;
  for (int c = 0; c < a.agg.n_vcols; ++c) fixed = fixed || (a.agg.vcol[c].flags & VF_FIXED) != 0;
  if (!a.sel && a.stage.n == 0 && a.agg.n_vcols <= QM_SPEC_NV_MAX && !fixed) {
    int kk = key_kind(a.key);
    if (kk == QM_KK_NONE && !dd) kk = QM_KK_ANY;
    switch (a.agg.n_vcols) {
      case 0: return qm_scan_nv0_launch(a, dd, kk, blocks, smem_bytes, st);
      case 1: return qm_scan_nv1_launch(a, dd, kk, blocks, smem_bytes, st);
      case 2: return qm_scan_nv2_launch(a, dd, kk, blocks, smem_bytes, st);
      case 3: return qm_scan_nv3_launch(a, dd, kk, blocks, smem_bytes, st);
      case 4: return qm_scan_nv4_launch(a, dd, kk, blocks, smem_bytes, st);
    }
  }
  if (a.sel) {
    if (dd) qm_scan_kernel<true, false, 1, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
    else qm_scan_kernel<true, false, 0, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
  } else if (a.stage.n > 0) {
    if (dd) qm_scan_kernel<false, true, 1, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
    else qm_scan_kernel<false, true, 0, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
  } else {
    if (dd) qm_scan_kernel<false, false, 1, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
    else qm_scan_kernel<false, false, 0, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem_bytes, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t qm_launch_init_table(uint64_t *t, int64_t n_slots_total, int stride, int hash_keys,
                                 const qm_aggspec &A, int sm_count, cudaStream_t st) {
  int64_t n = n_slots_total * stride;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 16);
  if (blocks < 1) blocks = 1;
  qm_init_table<<<blocks, 256, 0, st>>>(t, n_slots_total, stride, hash_keys, A);
  return cudaGetLastError();
}

cudaError_t qm_launch_compact(const uint64_t *t, int64_t n_slots_total, int stride, int count_word,
                              int first_word, uint64_t *keys_out, uint32_t *slots_out,
                              unsigned long long *counter, int sm_count, cudaStream_t st) {
  int blocks = (int)std::min<int64_t>((n_slots_total + 255) / 256, (int64_t)sm_count * 8);
  if (blocks < 1) blocks = 1;
  qm_compact_groups<<<blocks, 256, 0, st>>>(t, n_slots_total, stride, count_word, first_word, keys_out,
                                            slots_out, counter);
  return cudaGetLastError();
}

cudaError_t qm_sort_pairs(void *temp, size_t *temp_bytes, const uint64_t *kin, uint64_t *kout,
                          const uint32_t *vin, uint32_t *vout, int64_t n, int end_bit, cudaStream_t st) {
  return cub::DeviceRadixSort::SortPairs(temp, *temp_bytes, kin, kout, vin, vout, (int)n, 0, end_bit, st);
}

cudaError_t qm_launch_emit(const uint64_t *t, int stride, const uint32_t *slots, int64_t G,
                           const qm_keyspec &K, int64_t n_slots, const qm_outspec &O, unsigned char *out,
                           int sm_count, cudaStream_t st) {
  if (G <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((G + 255) / 256, (int64_t)sm_count * 8);
  qm_emit_groups<<<blocks, 256, 0, st>>>(t, stride, slots, G, K, n_slots, O, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_select_masks(const qm_pred &P, int64_t n, const uint32_t *sel, uint32_t *masks,
                                   uint32_t *counts, int sm_count, cudaStream_t st) {
  int64_t n_tiles = (n + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  int warps = QM_SCAN_THREADS / 32;
  int blocks = (int)std::min<int64_t>((n_tiles + warps - 1) / warps, (int64_t)sm_count * 4);
  if (blocks < 1) return cudaSuccess;
  if (sel) qm_select_masks<true><<<blocks, QM_SCAN_THREADS, 0, st>>>(P, n, sel, masks, counts);
  else qm_select_masks<false><<<blocks, QM_SCAN_THREADS, 0, st>>>(P, n, sel, masks, counts);
  return cudaGetLastError();
}

cudaError_t qm_launch_pq_decode(const uint8_t *chunk, const qm_pq_page *pages, int n_pages, const qm_pq_run *runs,
                                int n_runs, const qm_pq_run *iruns, int width, int in_width, int conv, int64_t n_rows, uint32_t *present, uint32_t *counts,
                                uint64_t *ranks, void *temp, size_t *temp_bytes, unsigned char *out, uint32_t *nulls,
                                int sm_count, cudaStream_t st) {
  const int64_t words = (n_rows + 31) / 32;
  if (!temp) {
    *temp_bytes = qm_scan_temp_bytes_for(words);
    return cudaSuccess;
  }
  if (n_rows <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((words + 255) / 256, (int64_t)sm_count * 8);
  // one resident wave: every warp owns a fixed range of words
  // variants: PLAIN, dictionary pages (Parquet), widened page values (Lance
  // pages only, so never with dictionary pages)
  static int occ_present = 0, occ_scatter[3] = {0, 0, 0};
  if (!occ_present) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_present, qm_pq_present, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_scatter[0], qm_pq_scatter<false, false>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_scatter[1], qm_pq_scatter<true, false>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_scatter[2], qm_pq_scatter<false, true>, 256, 0);
    occ_present = std::max(occ_present, 1);
    for (int &o : occ_scatter) o = std::max(o, 1);
  }
  const bool dict = iruns != nullptr;
  const bool wide = conv != 0;
  if (dict && wide) return cudaErrorInvalidValue;
  const int var = dict ? 1 : (wide ? 2 : 0);
  const auto scatter =
      dict ? qm_pq_scatter<true, false> : (wide ? qm_pq_scatter<false, true> : qm_pq_scatter<false, false>);
  const int pblocks = (int)std::min<int64_t>((words + 7) / 8, (int64_t)sm_count * occ_present);
  const int wblocks = (int)std::min<int64_t>((words + 7) / 8, (int64_t)sm_count * occ_scatter[var]);
  if (n_runs == 0) {  // no levels: every row present, values by row
    scatter<<<wblocks, 256, 0, st>>>(chunk, pages, n_pages, iruns, width, in_width, conv, n_rows, nullptr, nullptr, out,
                                     nulls);
    return cudaGetLastError();
  }
  qm_pq_present<<<pblocks, 256, 0, st>>>(chunk, pages, n_pages, runs, n_rows, present);
  (void)counts;
  (void)blocks;
  cudaError_t e = qm_scan_u64<true>(present, words, ranks, temp, *temp_bytes, st);
  if (e != cudaSuccess) return e;
  scatter<<<wblocks, 256, 0, st>>>(chunk, pages, n_pages, iruns, width, in_width, conv, n_rows, present, ranks, out,
                                   nulls);
  return cudaGetLastError();
}

cudaError_t qm_launch_zone_stats(const void *p, int dtype, const uint32_t *nulls, int64_t n, int64_t *zmin,
                                 int64_t *zmax, int64_t *zcount, cudaStream_t st) {
  const int64_t zones = (n + QM_ZONE_ROWS - 1) / QM_ZONE_ROWS;
  if (zones <= 0) return cudaSuccess;
  qm_zone_stats<<<(unsigned)zones, 512, 0, st>>>(p, dtype, nulls, n, zmin, zmax, zcount);
  return cudaGetLastError();
}

cudaError_t qm_launch_sort_keys(const unsigned char *data, const uint32_t *nulls, int dtype, int desc, int64_t G,
                                uint32_t *last, uint64_t *hi, uint64_t *lo, uint32_t *idx, int sm_count, cudaStream_t st) {
  if (G <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((G + 255) / 256, (int64_t)sm_count * 8);
  qm_sort_keys<<<blocks, 256, 0, st>>>(data, nulls, dtype, desc, G, last, hi, lo, idx);
  return cudaGetLastError();
}

// Stable sort of result rows by (last, hi, lo): LSD passes of stable radix
// sorts, each keyed by the next more significant word in the current order.
// idx holds 0..G-1 on entry and the sorted order on exit; tmp* are scratch of
// G elements.
cudaError_t qm_stable_sort_rows(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, bool wide, int64_t G,
                                uint32_t *idx, uint32_t *idx2, uint64_t *k1, uint64_t *k2, uint32_t *l1, uint32_t *l2,
                                void *temp, size_t *temp_bytes, int sm_count, cudaStream_t st) {
  size_t need = 0, t2 = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, need, k1, k2, idx, idx2, (int)G, 0, 64, st);
  if (e != cudaSuccess) return e;
  e = cub::DeviceRadixSort::SortPairs(nullptr, t2, l1, l2, idx, idx2, (int)G, 0, 1, st);
  if (e != cudaSuccess) return e;
  need = std::max(need, t2);
  if (!temp) {
    *temp_bytes = need;
    return cudaSuccess;
  }
  if (G <= 1) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((G + 255) / 256, (int64_t)sm_count * 8);
  const uint64_t *words[2] = {lo, wide ? hi : nullptr};
  for (int p = 0; p < 2; ++p) {
    if (!words[p]) continue;
    qm_gather_u64<<<blocks, 256, 0, st>>>(words[p], idx, G, k1);
    size_t tb = *temp_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, k1, k2, idx, idx2, (int)G, 0, 64, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(idx, idx2, sizeof(uint32_t) * G, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
  }
  qm_gather_u32<<<blocks, 256, 0, st>>>(last, idx, G, l1);
  size_t tb = *temp_bytes;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, l1, l2, idx, idx2, (int)G, 0, 1, st)) != cudaSuccess) return e;
  return cudaMemcpyAsync(idx, idx2, sizeof(uint32_t) * G, cudaMemcpyDeviceToDevice, st);
}

cudaError_t qm_launch_topk(const uint32_t *last, const uint64_t *hi, const uint64_t *lo, int64_t G, int64_t k,
                           uint32_t *heap, uint32_t *out, cudaStream_t st) {
  qm_topk_heap<<<1, QM_TOPK_THREADS, 0, st>>>(last, hi, lo, G, k, heap, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_gather_rows(const unsigned char *src, const qm_outspec &O, const qm_outspec &O2,
                                  const uint32_t *idx, int64_t first, int64_t n, unsigned char *dst, int sm_count,
                                  cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 8);
  qm_gather_rows<<<blocks, 256, 0, st>>>(src, O, O2, idx, first, n, dst);
  return cudaGetLastError();
}


cudaError_t qm_launch_rank_first(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                 uint32_t *bitmap, int64_t words, uint32_t *counts, uint64_t *ranks, void *temp,
                                 size_t temp_bytes, int sm_count, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(bitmap, 0, sizeof(uint32_t) * (size_t)(words + 1), st);
  if (e != cudaSuccess) return e;
  int blocks = (int)std::min<int64_t>((n_slots_total + 255) / 256, (int64_t)sm_count * 8);
  qm_mark_first<<<std::max(blocks, 1), 256, 0, st>>>(t, n_slots_total, stride, count_word, first_word, bitmap, words);
  // the words' popcounts go straight into the scan (no counts pass)
  (void)counts;
  return qm_scan_u64<true>(bitmap, words, ranks, temp, temp_bytes, st);
}

cudaError_t qm_rank_temp_bytes(int64_t words, size_t *bytes) {
  *bytes = qm_scan_temp_bytes_for(words);
  return cudaSuccess;
}

cudaError_t qm_launch_emit_ranked(const uint64_t *t, int64_t n_slots_total, int stride, int count_word,
                                  int first_word, const uint32_t *bitmap, const uint64_t *ranks, int64_t words,
                                  const qm_keyspec &K, int64_t n_slots, const qm_outspec &O, unsigned char *out,
                                  int sm_count, cudaStream_t st) {
  const int blocks = (int)std::min<int64_t>((n_slots_total + 255) / 256, (int64_t)sm_count * 8);
  qm_emit_ranked<<<std::max(blocks, 1), 256, 0, st>>>(t, n_slots_total, stride, count_word, first_word, bitmap, ranks,
                                                      words, K, n_slots, O, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_emit_walk(const qm_scan_args &a, const uint32_t *bitmap, const uint64_t *ranks, int64_t words,
                                const qm_outspec &O, unsigned char *out, int sm_count, cudaStream_t st,
                                const int64_t *bounds, int chunk) {
  const int blocks = (int)std::min<int64_t>((words + 255) / 256, (int64_t)sm_count * 8);
  qm_emit_walk<<<std::max(blocks, 1), 256, 0, st>>>(a, bitmap, ranks, words, O, out, bounds, chunk);
  return cudaGetLastError();
}

cudaError_t qm_launch_emit_perm(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                const uint32_t *bitmap, const uint64_t *ranks, int64_t words, uint32_t *perm,
                                int64_t rows, const qm_keyspec &K, int64_t n_slots, const qm_outspec &O,
                                unsigned char *out, int sm_count, cudaStream_t st) {
  const int b1 = (int)std::min<int64_t>((n_slots_total + 255) / 256, (int64_t)sm_count * 8);
  qm_rank_slots<<<std::max(b1, 1), 256, 0, st>>>(t, n_slots_total, stride, count_word, first_word, bitmap, ranks, words,
                                                  perm);
  const int b2 = (int)std::min<int64_t>((rows + 255) / 256, (int64_t)sm_count * 8);
  qm_emit_perm<<<std::max(b2, 1), 256, 0, st>>>(t, stride, perm, ranks, words, rows, K, n_slots, O, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_rank_small(const uint64_t *t, int64_t n_slots_total, int stride, int count_word, int first_word,
                                 uint32_t *perm, uint64_t *groups, cudaStream_t st) {
  if (n_slots_total > QM_SMALL_RANK_SLOTS) return cudaErrorInvalidValue;
  qm_rank_small<<<1, 1024, 0, st>>>(t, n_slots_total, stride, count_word, first_word, perm, groups);
  return cudaGetLastError();
}

cudaError_t qm_launch_emit_sorted(const uint64_t *t, int stride, const uint32_t *perm, const uint64_t *groups,
                                  int64_t rows, const qm_keyspec &K, int64_t n_slots, const qm_outspec &O,
                                  unsigned char *out, int sm_count, cudaStream_t st) {
  const int b = (int)std::min<int64_t>((rows + 255) / 256, (int64_t)sm_count * 8);
  qm_emit_perm<<<std::max(b, 1), 256, 0, st>>>(t, stride, perm, groups, 0, rows, K, n_slots, O, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_walk_bounds(const uint64_t *ranks, int64_t words, int64_t per, int chunks, int64_t *bounds,
                                  cudaStream_t st) {
  if (chunks < 1 || chunks > 1023) return cudaErrorInvalidValue;
  qm_walk_bounds<<<1, chunks + 1, 0, st>>>(ranks, words, per, chunks, bounds);
  return cudaGetLastError();
}

// Exclusive scan of n u32 counts into u64 offsets (out[n - 1] + in[n - 1]
// lands in out[n]).  temp null: *temp_bytes receives the scratch size.
cudaError_t qm_exclusive_scan_u32(void *temp, size_t *temp_bytes, const uint32_t *in, uint64_t *out, int64_t n,
                                  cudaStream_t st) {
  if (!temp) {
    *temp_bytes = qm_scan_temp_bytes_for(n);
    return cudaSuccess;
  }
  return qm_scan_u64<false>(in, n, out, temp, *temp_bytes, st, false);
}

cudaError_t qm_launch_select_write(int64_t n_tiles, const uint32_t *sel, const uint32_t *masks,
                                   const uint64_t *offsets, uint32_t *out, int64_t max_out, int sm_count,
                                   cudaStream_t st) {
  int warps = 256 / 32;
  int blocks = (int)std::min<int64_t>((n_tiles + warps - 1) / warps, (int64_t)sm_count * 8);
  if (blocks < 1) return cudaSuccess;
  qm_select_write<<<blocks, 256, 0, st>>>(n_tiles, sel, masks, offsets, out, max_out);
  return cudaGetLastError();
}

cudaError_t qm_launch_check_selection(const uint32_t *sel, int64_t n_sel, int64_t n_rows, qm_status *st,
                                      int sm_count, cudaStream_t stream) {
  if (n_sel <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((n_sel + 255) / 256, (int64_t)sm_count * 4);
  qm_check_selection<<<blocks, 256, 0, stream>>>(sel, n_sel, n_rows, st);
  return cudaGetLastError();
}

cudaError_t qm_launch_export_partial(const uint64_t *t, int stride, const uint32_t *slots, int64_t G, int64_t n_slots,
                                     int key_mode, const qm_aggspec &A, int64_t row_offset, uint64_t *dst, int sm_count,
                                     cudaStream_t st) {
  if (G <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((G + 255) / 256, (int64_t)sm_count * 8);
  qm_export_partial<<<blocks, 256, 0, st>>>(t, stride, slots, G, n_slots, key_mode, A, row_offset, dst);
  return cudaGetLastError();
}

cudaError_t qm_launch_partition_count(const uint64_t *src, int64_t n, int rw, int parts, unsigned long long *counts,
                                      int sm_count, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 4);
  qm_partition_count<<<blocks, 256, parts * sizeof(unsigned long long), st>>>(src, n, rw, parts, counts);
  return cudaGetLastError();
}

cudaError_t qm_launch_partition_scatter(const uint64_t *src, int64_t n, int rw, int parts, unsigned long long *cursor,
                                        uint64_t *dst, int sm_count, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 8);
  qm_partition_scatter<<<blocks, 256, 0, st>>>(src, n, rw, parts, cursor, dst);
  return cudaGetLastError();
}

cudaError_t qm_launch_merge_partial(const qm_scan_args &a, const uint64_t *src, int64_t n, int sm_count,
                                    cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 8);
  qm_merge_partial<<<blocks, 256, 0, st>>>(a, src, n);
  return cudaGetLastError();
}

cudaError_t qm_launch_sample_pred(const qm_pred &P, int64_t n, int n_samples, unsigned long long *count,
                                  cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess || n <= 0 || n_samples <= 0) return e;
  qm_sample_pred<<<(n_samples + 255) / 256, 256, 0, st>>>(P, n, n_samples, count);
  return cudaGetLastError();
}

cudaError_t qm_launch_hll(const qm_keyspec &K, int64_t n, uint32_t *regs, int sm_count, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(regs, 0, sizeof(uint32_t) << QM_HLL_P, st);
  if (e != cudaSuccess || n <= 0) return e;
  int blocks = (int)std::min<int64_t>((n + 1023) / 1024, (int64_t)sm_count * 2);
  qm_hll_kernel<<<blocks, 512, 0, st>>>(K, n, regs);
  return cudaGetLastError();
}

cudaError_t qm_launch_rehash(const uint64_t *old_t, int64_t old_cap, int stride, int count_word, uint64_t *new_t,
                             int log2cap, qm_status *st, int sm_count, cudaStream_t stream) {
  if (old_cap <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((old_cap + 255) / 256, (int64_t)sm_count * 8);
  qm_rehash<<<blocks, 256, 0, stream>>>(old_t, old_cap, stride, count_word, new_t, log2cap, st);
  return cudaGetLastError();
}

cudaError_t qm_launch_maxabs(const void *p, int dtype, const uint32_t *nulls, int64_t n, unsigned long long *out,
                             int sm_count, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, 8, st);
  if (e != cudaSuccess || n <= 0) return e;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 4);
  qm_maxabs_kernel<<<blocks, 256, 0, st>>>(p, dtype, nulls, n, out);
  return cudaGetLastError();
}

cudaError_t qm_launch_minmax(const void *p, int dtype, const uint32_t *nulls, int64_t n, long long *out,
                             int sm_count, cudaStream_t st) {
  qm_minmax_init<<<1, 1, 0, st>>>(out);
  if (n > 0) {
    int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 4);
    qm_minmax_kernel<<<blocks, 256, 0, st>>>(p, dtype, nulls, n, out);
  }
  return cudaGetLastError();
}
