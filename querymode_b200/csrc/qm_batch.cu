// qm_batch.cu — many filter -> GROUP BY queries in one persistent launch.
//
// Each query of a batch has its own plan (qm_scan_args), group table and
// status in device memory.  Work is cut into chunks (query, tile range);
// every block claims chunks from an atomic counter, keeps the current
// query's plan in shared memory, and merges its block-local table into the
// query's global table whenever it moves to another query.
//
// Finalize is batched too and needs no sort: a group's first-seen rank is
// the number of groups of its query whose first row is smaller, i.e. the
// prefix popcount of the query's bitmap of first rows at the group's own
// first row.  Each query's rows are written in that order (slot numbers
// scattered to their ranks, then rows emitted in order) into one packed
// buffer (columns, then NULL bitmaps), so one copy returns every result.
#include "qm_batch.h"
#include "qm_launch.h"
#include "qm_kernels.cuh"

namespace qm {

__device__ __forceinline__ int find_query(const int64_t *slot0, int n, int64_t gs) {
  int lo = 0, hi = n - 1;  // last query whose slot0 <= gs
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (slot0[mid] <= gs) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Each warp clears 32 consecutive slots (of one query or two): the lanes
// write consecutive words of the slots, so the stores are coalesced, and the
// query is looked up once per warp.
__global__ void qm_batch_init(const qm_bq *bq, const int64_t *slot0, int n, int64_t total) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t g = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; g < total; g += warps * 32) {
    const int64_t g1 = min(total, g + 32);
    int q = find_query(slot0, n, g);
    for (int64_t s0 = g; s0 < g1;) {
      while (q + 1 < n && slot0[q + 1] <= s0) ++q;
      const int64_t qend = q + 1 < n ? slot0[q + 1] : total;
      const int64_t s1 = min(g1, qend);
      const qm_scan_args &a = bq[q].a;
      const int stride = a.stride;
      uint64_t *base = a.table + (s0 - slot0[q]) * stride;
      const uint64_t key0 = a.key.mode == QK_HASH ? QM_EMPTY_KEY : 0ULL;
      const int nw = (int)(s1 - s0) * stride;  // at most 32 slots
      for (int j = lane; j < nw; j += 32) {
        const int w = j % stride;
        base[j] = w == 0 ? key0 : a.agg.init[w - 1];
      }
      s0 = s1;
    }
  }
}

// Shared memory: block-local table (keys, then words SoA), per-warp queues,
// per-warp merge scratch — sized for the batch's largest local table.
struct bsmem {
  size_t words_off, queue_off, scratch_off, bytes;
};
__host__ __device__ inline bsmem batch_smem(int local_bytes, int warps) {
  bsmem s;
  s.words_off = 0;
  s.queue_off = ((size_t)local_bytes + 15) & ~(size_t)15;
  s.scratch_off = s.queue_off + (size_t)warps * (QM_TILE_ROWS + 32) * sizeof(uint32_t);
  s.bytes = s.scratch_off + (size_t)warps * 64 * sizeof(uint64_t);
  return s;
}

__device__ void batch_flush(const qm_scan_args &a, uint64_t *lkeys, uint64_t *lw) {
  const int L = a.local_slots;
  if (L <= 0) return;
  const qm_aggspec &A = a.agg;
  for (int s = threadIdx.x; s < L; s += blockDim.x) {
    if (lw[(int64_t)A.w_count * L + s] == 0) continue;
    int64_t gs;
    if (a.local_hash) gs = global_slot(a, lkeys[s], 0);
    else gs = s;
    if (gs < 0) continue;
    merge_local(A, lw + s, L, a.table + gs * a.stride + 1);
  }
}

// DD / NV / KK: the dedupe flag, value-column count and key kind of the
// queries this instantiation takes (QM_NV_ANY / QM_KK_ANY / DD 2: read from
// each query's plan); a batch runs one persistent launch per class present.
template <int DD, int NV, int KK>
__global__ void __launch_bounds__(QM_SCAN_THREADS)
    qm_batch_scan(const qm_bq *__restrict__ bq, const qm_chunk *__restrict__ chunks, int n_chunks, int *counter,
                  int local_bytes) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ qm_scan_args P;
  __shared__ int s_chunk;
  __shared__ int l_used;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const bsmem lay = batch_smem(local_bytes, warps);
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem + lay.queue_off) + warp * (QM_TILE_ROWS + 32);
  uint64_t *scr = reinterpret_cast<uint64_t *>(smem + lay.scratch_off) + warp * 64;
  uint64_t *lkeys = reinterpret_cast<uint64_t *>(smem);
  uint64_t *lw = lkeys;
  int cur = -1;
  unsigned long long selected = 0;

  for (;;) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1);
    __syncthreads();
    const int c = s_chunk;
    if (c >= n_chunks) break;
    const qm_chunk ch = chunks[c];
    if (ch.q != cur) {
      if (cur >= 0) {
        batch_flush(P, lkeys, lw);
        if (lane == 0 && selected) atomicAdd(&P.status->rows_selected, selected);
        selected = 0;
      }
      __syncthreads();
      // load the next query's plan into shared memory
      const uint32_t *src = reinterpret_cast<const uint32_t *>(&bq[ch.q].a);
      uint32_t *dst = reinterpret_cast<uint32_t *>(&P);
      for (int i = threadIdx.x; i < (int)(sizeof(qm_scan_args) / 4); i += blockDim.x) dst[i] = __ldg(src + i);
      if (threadIdx.x == 0) l_used = 0;
      __syncthreads();
      const int L = P.local_slots;
      lw = lkeys + (P.local_hash ? L : 0);
      if (L > 0) {
        if (P.local_hash)
          for (int s = threadIdx.x; s < L; s += blockDim.x) lkeys[s] = QM_EMPTY_KEY;
        for (int i = threadIdx.x; i < L * P.agg.n_words; i += blockDim.x) lw[i] = P.agg.init[i / L];
      }
      __syncthreads();
      cur = ch.q;
    }
    const int L = P.local_slots;
    int qn = 0;
    for (int64_t tile = ch.tile0 + warp; tile < ch.tile1; tile += warps) {
      const int64_t e0 = tile * QM_TILE_ROWS;
      uint32_t m;
      const int64_t r0 = e0 + (int64_t)lane * QM_R;
      if (P.vec_ok && e0 + QM_TILE_ROWS <= P.n) {
        const int64_t nxt = tile + warps;
        if (nxt < ch.tile1 && (nxt + 1) * QM_TILE_ROWS <= P.n) prefetch_tile_l2(P.pred, nxt * QM_TILE_ROWS, lane);
        m = eval_pred_contig(P.pred, r0, (1u << QM_R) - 1);
      } else {
        int64_t rowv[QM_R];
        m = 0;
#pragma unroll
        for (int j = 0; j < QM_R; ++j) {
          m |= (uint32_t)(r0 + j < P.n) << j;
          rowv[j] = r0 + j;
        }
        auto rowf = [&](int j) { return rowv[j]; };
        m = eval_pred(P.pred, rowf, m);
      }
      const uint32_t cnt = __popc(m);
      uint32_t off = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(QM_FULL, off, o);
        if (lane >= o) off += x;
      }
      const uint32_t tot = __shfl_sync(QM_FULL, off, 31);
      uint32_t qp = qn + off - cnt;
      const uint32_t r0u = (uint32_t)r0;
      for (uint32_t mm = m; mm; mm &= mm - 1) queue[qp++] = r0u + (uint32_t)(__ffs(mm) - 1);
      qn += (int)tot;
      selected += tot;
      __syncwarp();
      while (qn >= 32) {
        const int64_t row = queue[qn - 32 + lane];
        __syncwarp();
        qn -= 32;
        drain_round_any<DD, NV, KK, (NV > QM_MAX_VCOLS)>(P, lkeys, lw, L, &l_used, lane, true, row, scr);
      }
    }
    if (qn > 0) {
      const bool active = lane < qn;
      const int64_t row = active ? (int64_t)queue[lane] : 0;
      __syncwarp();
      drain_round_any<DD, NV, KK, (NV > QM_MAX_VCOLS)>(P, lkeys, lw, L, &l_used, lane, active, row, scr);
    }
    __syncthreads();
  }
  if (cur >= 0) {
    batch_flush(P, lkeys, lw);
    if (lane == 0 && selected) atomicAdd(&P.status->rows_selected, selected);
  }
}

// Set bit `first row` of each occupied group in its query's bitmap.
// Slots go in warp-sized runs: a warp looks up the query of its run's first
// slot once, and each lane moves on to the query of its own slot.
__device__ __forceinline__ int run_query(const int64_t *slot0, int n, int64_t run, int64_t gs) {
  int q = find_query(slot0, n, run);
  while (q + 1 < n && slot0[q + 1] <= gs) ++q;
  return q;
}
#define QM_SLOT_RUNS(total)                                                                          \
  for (int64_t run = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; run < (total);    \
       run += (int64_t)gridDim.x * (blockDim.x >> 5) * 32)

__global__ void qm_batch_mark(const qm_bq *bq, const int64_t *slot0, int n, int64_t total, uint32_t *bitmap) {
  QM_SLOT_RUNS(total) {
    const int64_t gs = run + (threadIdx.x & 31);
    if (gs >= total) continue;
    const int q = run_query(slot0, n, run, gs);
    const qm_bq &b = bq[q];
    if (b.none) continue;
    const uint64_t *slot = b.a.table + (gs - slot0[q]) * b.a.stride + 1;
    if (slot[b.a.agg.w_count] == 0) continue;
    const uint64_t first = slot[b.a.agg.w_first];
    atomicOr(bitmap + b.bm_word0 + (int64_t)(first >> 5), 1u << (first & 31));
  }
}


__host__ __device__ inline int64_t align16(int64_t x) { return (x + 15) & ~(int64_t)15; }

// One block: each query's group count, its packed region and the offsets of
// its output columns, NULL byte maps and NULL bitmaps.  The queries go in
// chunks of blockDim.x, one per thread; a block-wide exclusive scan of their
// region sizes gives their bases.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t x, uint64_t *wsum, uint64_t &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  uint64_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(QM_FULL, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint64_t w = lane < nw ? wsum[lane] : 0;
    uint64_t z = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(QM_FULL, z, o);
      if (lane >= o) z += y;
    }
    if (lane < nw) wsum[lane] = z - w;
    if (lane == 31) wsum[32] = z;
  }
  __syncthreads();
  const uint64_t r = wsum[warp] + inc - x;
  total = wsum[32];
  __syncthreads();  // wsum is reused by the next chunk
  return r;
}

__global__ void __launch_bounds__(256) qm_batch_layout(qm_bq *bq, int n, const uint64_t *ranks, qm_batch_meta *meta) {
  __shared__ uint64_t wsum[33];
  uint64_t base = 0, nbase = 0;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int q = c0 + (int)threadIdx.x;
    int64_t G = 0, bytes = 0, nbytes = 0;
    if (q < n) {
      const qm_bq &b = bq[q];
      G = b.none ? 1 : (int64_t)(ranks[b.bm_word0 + b.bm_words] - ranks[b.bm_word0]);
      for (int k = 0; k < b.outs.n_out; ++k) {
        bytes += align16(G * b.width[k]);
        if (b.nullable[k]) {
          bytes += align16(((G + 31) / 32) * 4);
          nbytes += align16(G);
        }
      }
    }
    uint64_t tot, ntot;
    const uint64_t off0 = base + block_exclusive_scan((uint64_t)bytes, wsum, tot);
    const uint64_t noff0 = nbase + block_exclusive_scan((uint64_t)nbytes, wsum, ntot);
    if (q < n) {
      qm_bq &b = bq[q];
      meta->groups[q] = G;
      meta->base[q] = (int64_t)off0;
      meta->bytes[q] = bytes;
      int64_t off = (int64_t)off0, nb = (int64_t)noff0;
      for (int k = 0; k < b.outs.n_out; ++k) {
        b.outs.o[k].offset = off;
        off += align16(G * b.width[k]);
        if (b.nullable[k]) {
          b.outs.o[k].null_offset = off;  // packed bits (QMCB order)
          off += align16(((G + 31) / 32) * 4);
          b.nullbyte_off[k] = nb;
          nb += align16(G);
        } else {
          b.outs.o[k].null_offset = -1;
          b.nullbyte_off[k] = -1;
        }
      }
    }
    base += tot;
    nbase += ntot;
  }
  if (threadIdx.x == 0) {
    meta->total = (int64_t)base;
    meta->null_total = (int64_t)nbase;
  }
}

// Output order in two steps.  First, every occupied slot writes its slot
// number at its wave-wide first-seen rank (4-byte stores into an array that
// stays in L2); a query without GROUP BY writes its one row directly.
__global__ void qm_batch_order(const qm_bq *bq, const int64_t *slot0, int n, int64_t total, const uint32_t *bitmap,
                               const uint64_t *ranks, uint32_t *perm, unsigned char *packed,
                               unsigned char *nullbytes) {
  QM_SLOT_RUNS(total) {
    const int64_t gs = run + (threadIdx.x & 31);
    if (gs >= total) continue;
    const int q = run_query(slot0, n, run, gs);
    const qm_bq &b = bq[q];
    const int64_t s = gs - slot0[q];
    if (b.none) {
      if (s == 0)
        emit_group_bytes(b.a.table, b.a.stride, 0, 0, b.a.key, b.a.n_slots, b.outs, packed, nullbytes,
                         b.nullbyte_off);
      continue;
    }
    const uint64_t *slot = b.a.table + s * b.a.stride + 1;
    if (slot[b.a.agg.w_count] == 0) continue;
    const uint64_t first = slot[b.a.agg.w_first];
    const int64_t w = b.bm_word0 + (int64_t)(first >> 5);
    perm[ranks[w] + __popc(bitmap[w] & ((1u << (first & 31)) - 1u))] = (uint32_t)s;
  }
}

// Then each output row, in order, reads its group's slot: the output
// columns are written in runs instead of one scattered cell per column.
// Warps take 32 consecutive rows; the query of a row is the last one whose
// first rank is at or below it.
__global__ void qm_batch_emit_ordered(const qm_bq *bq, int n, const uint64_t *ranks, int64_t bm_words,
                                      const uint32_t *perm, unsigned char *packed, unsigned char *nullbytes) {
  const int lane = threadIdx.x & 31;
  const int64_t G = (int64_t)ranks[bm_words];
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < G; base += warps * 32) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((int64_t)ranks[bq[mid].bm_word0] <= base) lo = mid;
      else hi = mid - 1;
    }
    const int64_t o = base + lane;
    if (o >= G) continue;
    int q = lo;
    while (q + 1 < n && (int64_t)ranks[bq[q + 1].bm_word0] <= o) ++q;
    const qm_bq &b = bq[q];
    const int64_t i = o - (int64_t)ranks[b.bm_word0];
    emit_group_bytes(b.a.table, b.a.stride, (uint64_t)perm[o], i, b.a.key, b.a.n_slots, b.outs, packed, nullbytes,
                     b.nullbyte_off);
  }
}

// NULL byte maps -> QMCB bitmaps (one thread per 32 rows).
__global__ void qm_batch_pack_nulls(const qm_bq *bq, int n, const qm_batch_meta *meta, unsigned char *packed,
                                    const unsigned char *nullbytes) {
  const int q = blockIdx.y;
  if (q >= n) return;
  const qm_bq &b = bq[q];
  const int64_t G = meta->groups[q];
  const int64_t words = (G + 31) / 32;
  for (int k = 0; k < b.outs.n_out; ++k) {
    if (!b.nullable[k]) continue;
    const unsigned char *src = nullbytes + b.nullbyte_off[k];
    uint32_t *dst = reinterpret_cast<uint32_t *>(packed + b.outs.o[k].null_offset);
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (int64_t)gridDim.x * blockDim.x) {
      uint32_t bits = 0;
      for (int i = 0; i < 32; ++i) {
        const int64_t r = w * 32 + i;
        if (r < G && src[r]) bits |= 1u << i;
      }
      dst[w] = bits;
    }
  }
}

}  // namespace qm

using namespace qm;

size_t qm_batch_smem_bytes(int local_bytes) { return batch_smem(local_bytes, QM_SCAN_THREADS / 32).bytes; }

namespace {

template <int DD, int NV, int KK>
cudaError_t batch_class_configure(size_t attr_smem, size_t smem, int *blocks_per_sm) {
  cudaError_t e = cudaSuccess;
  if (attr_smem)
    e = cudaFuncSetAttribute(qm_batch_scan<DD, NV, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)attr_smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, qm_batch_scan<DD, NV, KK>, QM_SCAN_THREADS,
                                                       smem);
}

// The class instantiations: value-column counts 1 and 2 and key kinds int32 /
// int64 specialised, everything else through the run-time-plan kernel.
#define QM_BATCH_CLASSES(X)                                                                              \
  X(0, 1, QM_KK_I32) X(0, 1, QM_KK_I64) X(0, 2, QM_KK_I32) X(0, 2, QM_KK_I64) X(1, 1, QM_KK_I32)         \
  X(1, 1, QM_KK_I64) X(1, 2, QM_KK_I32) X(1, 2, QM_KK_I64)

}  // namespace

int qm_batch_class_of(const qm_scan_args &a) {
  bool fixed = false;
  for (int c = 0; c < a.agg.n_vcols; ++c) fixed = fixed || (a.agg.vcol[c].flags & VF_FIXED) != 0;
  const qm_keyspec &K = a.key;
  int kk = QM_KK_ANY;
  if (K.n_cols == 1 && K.pack == QP_RAW && K.nulls[0] == nullptr)
    kk = K.dtype[0] == QM_I64 ? QM_KK_I64 : K.dtype[0] == QM_I32 ? QM_KK_I32 : QM_KK_ANY;
  const int nv = a.agg.n_vcols;
  if (!fixed && (nv == 1 || nv == 2) && kk != QM_KK_ANY)
    return 1 + (a.dedupe ? 4 : 0) + (nv == 2 ? 2 : 0) + (kk == QM_KK_I64 ? 1 : 0);
  return 0;  // the run-time-plan kernel
}

cudaError_t qm_batch_class_configure(int cls, size_t attr_smem, size_t smem, int *blocks_per_sm) {
  int c = 1;
#define QM_CFG_(DD, NV, KK) \
  if (cls == c++) return batch_class_configure<DD, NV, KK>(attr_smem, smem, blocks_per_sm);
  QM_BATCH_CLASSES(QM_CFG_)
#undef QM_CFG_
  return batch_class_configure<2, QM_NV_ANY, QM_KK_ANY>(attr_smem, smem, blocks_per_sm);
}

cudaError_t qm_batch_launch_class(int cls, const qm_bq *bq, const qm_chunk *chunks, int n_chunks, int *counter,
                                  int local_bytes, int blocks, size_t smem, cudaStream_t st) {
  int c = 1;
#define QM_LAUNCH_(DD, NV, KK)                                                                            \
  if (cls == c++) {                                                                                       \
    qm_batch_scan<DD, NV, KK><<<blocks, QM_SCAN_THREADS, smem, st>>>(bq, chunks, n_chunks, counter, local_bytes); \
    return cudaGetLastError();                                                                            \
  }
  QM_BATCH_CLASSES(QM_LAUNCH_)
#undef QM_LAUNCH_
  qm_batch_scan<2, QM_NV_ANY, QM_KK_ANY><<<blocks, QM_SCAN_THREADS, smem, st>>>(bq, chunks, n_chunks, counter,
                                                                              local_bytes);
  return cudaGetLastError();
}


static int grid_for(int64_t n, int sm_count, int per_sm) {
  int64_t b = (n + 255) / 256;
  b = std::min<int64_t>(b, (int64_t)sm_count * per_sm);
  return (int)std::max<int64_t>(b, 1);
}

cudaError_t qm_batch_launch_init(const qm_batch_dev &d, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(d.statuses, 0, sizeof(qm_status) * d.n, st))) return e;
  if ((e = cudaMemsetAsync(d.counter, 0, sizeof(int) * QM_BATCH_CLASS_SLOTS, st))) return e;
  if ((e = cudaMemsetAsync(d.bitmap, 0, sizeof(uint32_t) * (d.bm_words + 1), st))) return e;
  qm_batch_init<<<grid_for(d.total_slots, d.sm_count, 16), 256, 0, st>>>(d.bq, d.slot0, d.n, d.total_slots);
  return cudaGetLastError();
}

cudaError_t qm_batch_launch_finalize(const qm_batch_dev &d, cudaStream_t st) {
  cudaError_t e;
  qm_batch_mark<<<grid_for(d.total_slots, d.sm_count, 8), 256, 0, st>>>(d.bq, d.slot0, d.n, d.total_slots, d.bitmap);
  if ((e = qm_scan_popc_words(d.bitmap, d.bm_words, d.ranks, d.scan_temp, d.scan_temp_bytes, st))) return e;
  qm_batch_layout<<<1, 256, 0, st>>>(d.bq, d.n, d.ranks, d.meta);
  qm_batch_order<<<grid_for(d.total_slots, d.sm_count, 8), 256, 0, st>>>(d.bq, d.slot0, d.n, d.total_slots, d.bitmap,
                                                                          d.ranks, d.perm, d.packed, d.nullbytes);
  qm_batch_emit_ordered<<<grid_for(d.total_slots, d.sm_count, 8), 256, 0, st>>>(d.bq, d.n, d.ranks, d.bm_words, d.perm,
                                                                                 d.packed, d.nullbytes);
  dim3 pg(8, d.n);
  qm_batch_pack_nulls<<<pg, 128, 0, st>>>(d.bq, d.n, d.meta, d.packed, d.nullbytes);
  if ((e = cudaMemcpyAsync(d.meta_host, d.meta, d.meta_bytes, cudaMemcpyDeviceToHost, st))) return e;
  return cudaGetLastError();
}

cudaError_t qm_batch_scan_temp_bytes(int64_t words, size_t *bytes) {
  *bytes = qm_scan_temp_bytes_for(words);
  return cudaSuccess;
}
