// qm_scan.cuh — the fused filter + GROUP BY scan kernel template.  Its
// instantiations live in several translation units (qm_kernels.cu: the
// run-time-plan kernels; qm_scan_nv*.cu: kernels specialised for a value
// column count and key kind) so they compile in parallel.
#pragma once

#include "qm_kernels.cuh"
#include "qm_launch.h"

namespace qm {

// Shared memory of one block: the block-local group table (keys, then the
// accumulator words structure-of-arrays), then one survivor queue per warp.
#define QM_WQ (QM_TILE_ROWS + 32)  // per-warp queue: a tile's survivors + < 32 left over

struct smem_layout {
  int L;
  size_t keys_off, words_off, queue_off, scratch_off, stage_off, stage_warp_bytes, bytes;
};

// Per warp staging region: QM_STAGE_MAX_DEPTH mbarriers (32 bytes), then
// `depth` tile buffers of tile_bytes each.
__host__ __device__ inline smem_layout make_smem_layout(int local_slots, int local_hash, int n_words, int warps,
                                                        int stage_tile_bytes = 0, int stage_depth = 0, int priv = 0) {
  smem_layout s;
  s.L = local_slots;
  s.keys_off = 0;
  size_t kb = (local_slots > 0 && local_hash) ? (size_t)local_slots * 8 : 0;
  s.words_off = kb;
  size_t wb = (size_t)local_slots * n_words * 8 * (priv ? warps : 1);  // priv: one copy per warp
  s.queue_off = (s.words_off + wb + 15) & ~(size_t)15;
  s.scratch_off = (s.queue_off + (size_t)warps * QM_WQ * sizeof(uint32_t) + 15) & ~(size_t)15;
  s.stage_off = (s.scratch_off + (size_t)warps * 64 * sizeof(uint64_t) + 127) & ~(size_t)127;
  s.stage_warp_bytes = stage_depth > 0 ? (size_t)(32 + stage_depth * stage_tile_bytes + 127) & ~(size_t)127 : 0;
  s.bytes = s.stage_off + (size_t)warps * s.stage_warp_bytes;
  return s;
}

template <bool SEL, int DD, int NV, int KK>
__device__ __forceinline__ void drain_round(const qm_scan_args &a, uint64_t *lkeys, uint64_t *lw, int L,
                                            int *l_used, int lane, bool active, int64_t row, uint64_t *scr) {
  // the fixed-point sum paths only in the run-time-plan kernels
  drain_round_any<DD, NV, KK, (NV > QM_MAX_VCOLS)>(a, lkeys, lw, L, l_used, lane, active, row, scr);
}

// The fused scan.  Each warp takes tiles of QM_TILE_ROWS rows round robin,
// filters them, appends the survivors' row indices to its own queue in
// shared memory and aggregates 32 survivors at a time (one per lane): gather
// the key and value cells, find the slot in the block-local table (else the
// global table) and update the accumulators.  With STAGED, the filter
// columns of the warp's next tiles stream into its shared-memory buffers by
// bulk async copies (lane 0 issues, an mbarrier per buffer counts the bytes)
// while the current tile is evaluated.
// NV / KK: the value-column count and key kind the kernel is specialised
// for (QM_NV_ANY / QM_KK_ANY: read from the plan at run time).
template <bool SEL, bool STAGED, int DD, int NV, int KK>
__global__ void __launch_bounds__(QM_SCAN_THREADS)
    qm_scan_kernel(const __grid_constant__ qm_scan_args a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const qm_aggspec &A = a.agg;
  const qm_staging &S = a.stage;
  const smem_layout lay =
      make_smem_layout(a.local_slots, a.local_hash, A.n_words, warps, STAGED ? S.tile_bytes : 0, STAGED ? S.depth : 0,
                       a.priv);
  const int L = lay.L;
  uint64_t *lkeys = reinterpret_cast<uint64_t *>(smem + lay.keys_off);
  uint64_t *lw = reinterpret_cast<uint64_t *>(smem + lay.words_off);
  // a private (per-warp) table: this warp's copy
  uint64_t *lwm = a.priv ? lw + (int64_t)warp * L * A.n_words : lw;
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem + lay.queue_off) + warp * QM_WQ;
  uint64_t *scr = reinterpret_cast<uint64_t *>(smem + lay.scratch_off) + warp * 64;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + lay.stage_off + warp * lay.stage_warp_bytes);
  uint8_t *sbuf = smem + lay.stage_off + warp * lay.stage_warp_bytes + 32;
  __shared__ int l_used;
  __shared__ unsigned long long blk_selected;

  if (threadIdx.x == 0) {
    l_used = 0;
    blk_selected = 0;
  }
  if (L > 0) {
    if (a.local_hash)
      for (int s = threadIdx.x; s < L; s += blockDim.x) lkeys[s] = QM_EMPTY_KEY;
    const int per = L * A.n_words;
    for (int i = threadIdx.x; i < per * (a.priv ? warps : 1); i += blockDim.x) lw[i] = A.init[(i % per) / L];
  }
  if (STAGED && lane == 0) {
    for (int d = 0; d < S.depth; ++d) mbar_init(&mbar[d], 1);
    fence_async_shared();
  }
  __syncthreads();

  const int64_t n_tiles = (a.n + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  const int64_t full_tiles = a.n / QM_TILE_ROWS;
  const int64_t gwarps = (int64_t)gridDim.x * warps;
  const int64_t first = (int64_t)blockIdx.x * warps + warp;
  const uint32_t lt = lanemask_lt();
  int qn = 0;  // warp-uniform queue length
  unsigned long long selected = 0;
  int64_t issued = 0;  // STAGED: tiles whose copies were issued (in order)
  bool failed = false;

  // lane 0 issues the copies of the warp's k-th tile into buffer k % depth
  auto issue = [&](int64_t k) {
    const int64_t tile = first + k * gwarps;
    if (tile >= full_tiles) return;
    if (lane == 0) {
      fence_async_shared();
      const int b = (int)(k % S.depth);
      uint8_t *dst = sbuf + b * S.tile_bytes;
      mbar_expect_tx(&mbar[b], (uint32_t)S.tile_bytes);
      for (int c = 0; c < S.n; ++c)
        bulk_g2s(dst + S.off[c], reinterpret_cast<const uint8_t *>(S.data[c]) + tile * QM_TILE_ROWS * S.elem[c],
                 (uint32_t)(QM_TILE_ROWS * S.elem[c]), &mbar[b]);
    }
    issued = k + 1;
  };
  if (STAGED)
    for (int64_t k = 0; k < S.depth - 1; ++k) issue(k);

  // with zone maps, virtual tile v walks the kept zones' tiles
  const int64_t n_virtual = a.zones ? a.n_zone_tiles : n_tiles;
  auto tile_of = [&](int64_t v) -> int64_t {
    return a.zones ? ((int64_t)a.zones[v / QM_ZONE_TILES] * QM_ZONE_TILES + v % QM_ZONE_TILES) : v;
  };
  int64_t k = 0;
  for (int64_t v = first; v < n_virtual; v += gwarps, ++k) {
    const int64_t tile = tile_of(v);
    if (tile >= n_tiles) continue;  // the table's last zone is partial
    const int64_t e0 = tile * QM_TILE_ROWS;
    uint32_t m = 0;
    if (STAGED && tile < full_tiles) {
      __syncwarp();
      issue(k + S.depth - 1);
      const int b = (int)(k % S.depth);
      if (!mbar_wait(&mbar[b], (uint32_t)((k / S.depth) & 1))) {
        set_error(a.status, QM_DEV_TIMEOUT);
        failed = true;
        break;
      }
      m = eval_pred_staged(a.pred, S, sbuf + b * S.tile_bytes, e0, lane, (1u << QM_R) - 1);
      // append survivors (rows e0 + j*32 + lane)
      uint32_t base = (uint32_t)qn;
#pragma unroll
      for (int j = 0; j < QM_R; ++j) {
        const uint32_t bal = __ballot_sync(QM_FULL, (m >> j) & 1);
        if ((m >> j) & 1) queue[base + __popc(bal & lt)] = (uint32_t)(e0 + j * 32 + lane);
        base += __popc(bal);
      }
      const int tot = (int)base - qn;
      qn = (int)base;
      selected += tot;
    } else if (!SEL && a.vec_ok && e0 + QM_TILE_ROWS <= a.n) {
      // full dense tile: the lane's rows are r0 .. r0+7
      const int64_t r0 = e0 + (int64_t)lane * QM_R;
      const int64_t nxt = v + gwarps < n_virtual ? tile_of(v + gwarps) * QM_TILE_ROWS : a.n;
      if (nxt + QM_TILE_ROWS <= a.n) {
        prefetch_tile_l2(a.pred, nxt, lane);
        if (QM_PREFETCH_PAYLOAD) prefetch_payload_l2<NV, KK>(a.key, A, nxt, lane);
      }
      m = eval_pred_contig(a.pred, r0, (1u << QM_R) - 1);
      const uint32_t cnt = __popc(m);
      uint32_t off = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(QM_FULL, off, o);
        if (lane >= o) off += x;
      }
      const uint32_t tot = __shfl_sync(QM_FULL, off, 31);
      uint32_t q = qn + off - cnt;
      const uint32_t r0u = (uint32_t)r0;
      for (uint32_t mm = m; mm; mm &= mm - 1) queue[q++] = r0u + (uint32_t)(__ffs(mm) - 1);
      qn += (int)tot;
      selected += tot;
    } else {
      const int64_t r0 = e0 + (int64_t)lane * QM_R;  // this lane's first element
      int64_t rowv[QM_R];
#pragma unroll
      for (int j = 0; j < QM_R; ++j) {
        const bool in = r0 + j < a.n;
        m |= (uint32_t)in << j;
        rowv[j] = r0 + j;
      }
      {
        if (SEL) {
#pragma unroll
          for (int j = 0; j < QM_R; ++j) rowv[j] = ((m >> j) & 1) ? (int64_t)__ldg(a.sel + r0 + j) : 0;
        }
        auto rowf = [&](int j) { return rowv[j]; };
        m = eval_pred(a.pred, rowf, m);
      }
      // append survivors (order inside the queue does not matter: FIRST is a min)
      const uint32_t cnt = __popc(m);
      uint32_t off = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(QM_FULL, off, o);
        if (lane >= o) off += x;
      }
      const uint32_t tot = __shfl_sync(QM_FULL, off, 31);
      off -= cnt;  // exclusive prefix
      uint32_t q = qn + off;
#pragma unroll
      for (int j = 0; j < QM_R; ++j)
        if ((m >> j) & 1) queue[q++] = (uint32_t)rowv[j];
      qn += (int)tot;
      selected += tot;
    }
    __syncwarp();
    while (qn >= 32) {
      const int64_t row = queue[qn - 32 + lane];
      __syncwarp();
      qn -= 32;
      drain_round<SEL, DD, NV, KK>(a, lkeys, lwm, L, &l_used, lane, true, row, scr);
    }
  }
  if (STAGED && failed) {
    // let every copy still in flight land before the block's memory goes
    for (int64_t j = k; j < issued; ++j)
      if (!mbar_wait(&mbar[j % S.depth], (uint32_t)((j / S.depth) & 1))) break;
  }
  if (qn > 0) {
    const bool active = lane < qn;
    const int64_t row = active ? (int64_t)queue[lane] : 0;
    __syncwarp();
    drain_round<SEL, DD, NV, KK>(a, lkeys, lwm, L, &l_used, lane, active, row, scr);
  }

  if (lane == 0 && selected) atomicAdd(&blk_selected, selected);
  __syncthreads();
  if (threadIdx.x == 0 && blk_selected) atomicAdd(&a.status->rows_selected, blk_selected);

  // merge the block-local table into the global table
  if (L > 0) {
    const int cw = A.w_count;
    if (a.priv) {  // fold the per-warp copies into copy 0
      for (int s = threadIdx.x; s < L; s += blockDim.x)
        for (int w = 1; w < warps; ++w) {
          const uint64_t *src = lw + (int64_t)w * L * A.n_words + s;
          if (src[(int64_t)cw * L] != 0) merge_plain(A, lw + s, src, L);
        }
      __syncthreads();
    }
    for (int s = threadIdx.x; s < L; s += blockDim.x) {
      const uint64_t *lp = lw + s;
      if (lp[(int64_t)cw * L] == 0) continue;
      int64_t gs;
      if (a.local_hash) gs = global_slot(a, lkeys[s], 0);
      else gs = s;
      if (gs < 0) continue;
      merge_local(A, lp, L, a.table + gs * a.stride + 1);
    }
  }
}

}  // namespace qm
