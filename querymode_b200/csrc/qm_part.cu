// qm_part.cu — partitioned aggregation for group tables larger than a
// block's shared memory (many groups, many selected rows).
//
// The fused scan updates the group table with one atomic per accumulator
// word per selected row; when the table lives in L2 or DRAM those atomics,
// not the column reads, set the pace.  Here the work is split instead:
//   1. counting pass: the scan's filter and compaction, then per survivor
//      its key's partition, counted per (partition, block) in shared memory;
//   2. offsets: each (partition, block)'s first record, partitions back to
//      back (a prefix over blocks per partition, then over partitions);
//   3. scatter pass: the same scan over the same rows (same grid, so every
//      block sees the same rows), each survivor written as a record at its
//      (partition, block)'s next place;
//   4. aggregation: blocks take chunks of the record array (contiguous,
//      coalesced reads) and aggregate each partition's records in a
//      shared-memory table — a window of the direct table or a hash table
//      of the partition's keys — with shared-memory updates, then merge
//      that table into the group table once per chunk.
// Every record of a group lands in one partition; a partition held whole by
// one chunk is written to its slots by plain stores.  First-seen order,
// exact integer sums and compensated float sums follow from the same
// accumulator code as the scan.  The partitions are kept few (at most 512)
// so that the scatter's open write lines, one per (partition, block), stay
// in L2 and reach DRAM as whole lines.
#include "qm_kernels.cuh"
#include "qm_launch.h"
#include "qm_scan.cuh"

#include <algorithm>
#include <mutex>

namespace qm {

__device__ __forceinline__ int part_of(const qm_scan_args &a, const qm_part_spec &ps, uint64_t key, int special) {
  if (special) return ps.parts;
  if (ps.direct) {
    const uint64_t d = key - (uint64_t)a.key.base;
    return d < (uint64_t)a.n_slots ? (int)(d >> ps.shift) : ps.parts;
  }
  return ps.bits > 0 ? (int)(fmix64(key ^ 0x5851f42d4c957f2dULL) >> (64 - ps.bits)) : 0;
}

// One survivor per lane: its partition counted (pass 0) or its record
// written (pass 1).  Lanes of a warp bound for one partition take
// consecutive places with one shared-memory atomic.
template <int PASS, int NV, int KK>
__device__ __forceinline__ void part_round(const qm_scan_args &a, const qm_part_spec &ps, uint32_t *cnt, int lane,
                                           bool active, int64_t row) {
  int special = 0;
  uint64_t key = 0;
  int p = 0;
  if (active) {
    key = row_key<KK>(a.key, row, special);
    p = part_of(a, ps, key, special);
  }
  const unsigned act = __ballot_sync(QM_FULL, active);
  if (!active) return;
  const unsigned peers = __match_any_sync(act, p);
  const int leader = __ffs(peers) - 1;
  uint32_t at = 0;
  if (lane == leader) at = atomicAdd(&cnt[p], (uint32_t)__popc(peers));
  at = __shfl_sync(peers, at, leader) + __popc(peers & ((1u << lane) - 1));
  if (PASS == 0) return;
  uint64_t vb[QM_MAX_VCOLS];
  uint32_t vnull;
  gather_values<NV>(a.agg, row, vb, vnull);
  const uint64_t pos = ps.bases[p] + ps.offsets[(int64_t)p * ps.blocks + blockIdx.x] + at;
  if (pos >= (uint64_t)ps.rec_cap) {  // more survivors than planned: regrow and run again
    set_error(a.status, QM_DEV_OVERFLOW);
    return;
  }
  // a record is a whole number of 32-byte sectors, written as 16-byte
  // stores: full sectors reach L2, so no partial sector goes back to DRAM
  ulonglong2 *rec = reinterpret_cast<ulonglong2 *>(ps.records + pos * ps.rec_words);
  const int nv = NV > QM_MAX_VCOLS ? a.agg.n_vcols : NV;
  uint64_t w[QM_MAX_VCOLS + 2];
  w[0] = key;
  w[1] = (uint64_t)(uint32_t)row | ((uint64_t)(uint32_t)special << 32) | ((uint64_t)vnull << 40);
#pragma unroll
  for (int c = 0; c < QM_MAX_VCOLS; ++c) w[2 + c] = c < QM_NV_BOUND(NV) && c < nv ? vget<NV>(vb, c) : 0;
#pragma unroll
  for (int k = 0; k < (QM_MAX_VCOLS + 2) / 2; ++k)
    if (2 * k < ps.rec_words) rec[k] = make_ulonglong2(w[2 * k], w[2 * k + 1]);
}

// Passes 0 and 1: the scan's tile walk and filter (every warp takes tiles
// round robin, so a block sees the same rows in both passes).
template <int PASS, int NV, int KK>
__global__ void __launch_bounds__(QM_SCAN_THREADS)
    qm_part_scan(const __grid_constant__ qm_scan_args a, const __grid_constant__ qm_part_spec ps) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem) + warp * QM_WQ;
  uint32_t *cnt = reinterpret_cast<uint32_t *>(smem) + warps * QM_WQ;  // parts + 1 counters
  __shared__ unsigned long long blk_selected;
  const int P1 = ps.parts + 1;
  for (int p = threadIdx.x; p < P1; p += blockDim.x) cnt[p] = 0;
  if (threadIdx.x == 0) blk_selected = 0;
  __syncthreads();
  const int64_t n_tiles = (a.n + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  const int64_t gwarps = (int64_t)gridDim.x * warps;
  const int64_t first = (int64_t)blockIdx.x * warps + warp;
  const int64_t n_virtual = a.zones ? a.n_zone_tiles : n_tiles;
  auto tile_of = [&](int64_t v) -> int64_t {
    return a.zones ? ((int64_t)a.zones[v / QM_ZONE_TILES] * QM_ZONE_TILES + v % QM_ZONE_TILES) : v;
  };
  int qn = 0;
  unsigned long long selected = 0;
  for (int64_t v = first; v < n_virtual; v += gwarps) {
    const int64_t tile = tile_of(v);
    if (tile >= n_tiles) continue;
    const int64_t e0 = tile * QM_TILE_ROWS;
    const int64_t r0 = e0 + (int64_t)lane * QM_R;
    uint32_t m;
    if (a.vec_ok && e0 + QM_TILE_ROWS <= a.n) {
      const int64_t nxt = v + gwarps < n_virtual ? tile_of(v + gwarps) * QM_TILE_ROWS : a.n;
      if (nxt + QM_TILE_ROWS <= a.n) prefetch_tile_l2(a.pred, nxt, lane);
      m = eval_pred_contig(a.pred, r0, (1u << QM_R) - 1);
    } else {
      int64_t rowv[QM_R];
      m = 0;
#pragma unroll
      for (int j = 0; j < QM_R; ++j) {
        m |= (uint32_t)(r0 + j < a.n) << j;
        rowv[j] = r0 + j;
      }
      auto rowf = [&](int j) { return rowv[j]; };
      m = eval_pred(a.pred, rowf, m);
    }
    const uint32_t c = __popc(m);
    uint32_t off = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x = __shfl_up_sync(QM_FULL, off, o);
      if (lane >= o) off += x;
    }
    const uint32_t tot = __shfl_sync(QM_FULL, off, 31);
    uint32_t q = qn + off - c;
    for (uint32_t mm = m; mm; mm &= mm - 1) queue[q++] = (uint32_t)r0 + (uint32_t)(__ffs(mm) - 1);
    qn += (int)tot;
    selected += tot;
    __syncwarp();
    while (qn >= 32) {
      const int64_t row = queue[qn - 32 + lane];
      __syncwarp();
      qn -= 32;
      part_round<PASS, NV, KK>(a, ps, cnt, lane, true, row);
    }
  }
  if (qn > 0) {
    const bool active = lane < qn;
    const int64_t row = active ? (int64_t)queue[lane] : 0;
    __syncwarp();
    part_round<PASS, NV, KK>(a, ps, cnt, lane, active, row);
  }
  if (PASS == 0) {
    if (lane == 0 && selected) atomicAdd(&blk_selected, selected);
    __syncthreads();
    if (threadIdx.x == 0 && blk_selected) atomicAdd(&a.status->rows_selected, blk_selected);
    for (int p = threadIdx.x; p < P1; p += blockDim.x) ps.counts[(int64_t)p * ps.blocks + blockIdx.x] = cnt[p];
  }
}

// Pass 2a: one warp per partition: each block's first record relative to
// the partition's start (an exclusive prefix over blocks, 32 at a time), and
// the partition's total into bases[p].
__global__ void qm_part_prefix(const __grid_constant__ qm_part_spec ps) {
  const int lane = threadIdx.x & 31;
  const int P1 = ps.parts + 1;
  const int B = ps.blocks;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = wid; p < P1; p += nw) {
    uint64_t carry = 0;
    for (int b0 = 0; b0 < B; b0 += 32) {
      const int b = b0 + lane;
      const uint64_t c = b < B ? ps.counts[p * B + b] : 0;
      uint64_t x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(QM_FULL, x, o);
        if (lane >= o) x += y;
      }
      if (b < B) ps.offsets[p * B + b] = carry + x - c;
      carry += __shfl_sync(QM_FULL, x, 31);
    }
    if (lane == 0) ps.bases[p] = carry;
  }
}

// Pass 2b, one block of 1024 threads: the partitions' totals into their
// first records (an exclusive prefix), then the total of all records.
__global__ void qm_part_bases(const __grid_constant__ qm_part_spec ps) {
  __shared__ uint64_t sums[1024];
  const int P1 = ps.parts + 1;
  const int per = (P1 + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per;
  uint64_t t = 0;
  for (int i = 0; i < per; ++i)
    if (b0 + i < P1) t += ps.bases[b0 + i];
  sums[threadIdx.x] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t acc = 0;
    for (int i = 0; i < (int)blockDim.x; ++i) {
      const uint64_t x = sums[i];
      sums[i] = acc;
      acc += x;
    }
    ps.bases[P1] = acc;
  }
  __syncthreads();
  uint64_t acc = sums[threadIdx.x];
  for (int i = 0; i < per; ++i)
    if (b0 + i < P1) {
      const uint64_t x = ps.bases[b0 + i];
      ps.bases[b0 + i] = acc;
      acc += x;
    }
}

// A partition's shared-memory table written into the group table by plain
// stores: the block holding every record of the partition owns its slots.
__device__ __forceinline__ void store_local(const qm_aggspec &A, const uint64_t *lp, int L, uint64_t *gp) {
  for (int i = 0; i < A.n_accs; i++) {
    const qm_acc ac = A.acc[i];
    const uint64_t v0 = lp[(int64_t)ac.word * L];
    uint64_t *g0 = gp + ac.word;
    if (ac.kind == QA_ISUM) {
      if (ac.wide) {
        g0[0] = v0;
        g0[1] = lp[(int64_t)(ac.word + 1) * L];
      } else if (ac.narrow) {
        g0[0] = v0;
      } else {  // a 64-bit block-local sum into the 128-bit table word pair
        g0[0] = v0;
        g0[1] = (int64_t)v0 < 0 ? ~0ULL : 0ULL;
      }
    } else if (ac.kind == QA_FSUM) {
      g0[0] = v0;
      g0[1] = lp[(int64_t)(ac.word + 1) * L];
    } else {
      g0[0] = v0;
    }
  }
}

// Pass 4: blocks claim chunks of `chunk` records of the record array (a
// large partition is shared by several blocks, a small one shares a chunk
// with its neighbours) and walk a chunk partition by partition: each
// partition's records go through a shared-memory table — the partition's
// window of a direct table, or a hash table of its keys (keys it does not
// admit go to the group table directly) — which is then merged into the
// group table: by plain stores when the chunk holds the whole partition of a
// direct table, else with atomics.  The last partition (special keys, direct
// keys outside the table) goes to the group table directly, where the scan's
// range check reports them.
template <int DD, int NV>
__global__ void __launch_bounds__(QM_SCAN_THREADS)
    qm_part_agg(const __grid_constant__ qm_scan_args a, const __grid_constant__ qm_part_spec ps, int64_t chunk) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ qm_scan_args P;
  __shared__ int s_chunk;
  __shared__ int l_used;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const qm_aggspec &A = a.agg;
  const int Lmax = ps.local_slots;
  const int hashed = ps.direct ? 0 : 1;
  uint64_t *lkeys = reinterpret_cast<uint64_t *>(smem);
  uint64_t *lw = lkeys + (hashed ? Lmax : 0);
  uint64_t *scr = reinterpret_cast<uint64_t *>(smem + (size_t)Lmax * 8 * (hashed + A.n_words)) + warp * 64;
  const int nv = NV > QM_MAX_VCOLS ? A.n_vcols : NV;
  const int P1 = ps.parts + 1;
  const uint64_t total = ps.bases[P1];
  for (;;) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(ps.counter, 1);
    __syncthreads();
    const uint64_t c0 = (uint64_t)s_chunk * (uint64_t)chunk;
    if (c0 >= total) break;
    const uint64_t c1 = min(total, c0 + (uint64_t)chunk);
    // the partition holding record c0: the last p with bases[p] <= c0
    int lo = 0, hi = P1 - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ps.bases[mid] <= c0) lo = mid;
      else hi = mid - 1;
    }
    for (int p = lo; p < P1; ++p) {
      const uint64_t pb = ps.bases[p], pe = ps.bases[p + 1];
      const uint64_t r0 = max(pb, c0), r1 = min(pe, c1);
      if (r0 >= c1) break;
      if (r0 >= r1) continue;
      const bool whole = pb >= c0 && pe <= c1;
      // this partition's plan: a window of the direct table, or the hash
      // table with a shared-memory front
      {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&a);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&P);
        for (int i = threadIdx.x; i < (int)(sizeof(qm_scan_args) / 4); i += blockDim.x) dst[i] = src[i];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        l_used = 0;
        P.priv = 0;
        if (p == ps.parts) {
          P.local_slots = 0;
        } else if (ps.direct) {
          const int64_t base = (int64_t)p << ps.shift;
          P.key.base = a.key.base + base;
          P.n_slots = min((int64_t)Lmax, a.n_slots - base);
          P.table = a.table + base * a.stride;
          P.local_slots = (int)P.n_slots;
          P.local_hash = 0;
        } else {
          P.local_slots = Lmax;
          P.local_hash = 1;
        }
      }
      __syncthreads();
      const int L = P.local_slots;
      if (L > 0) {
        if (hashed)
          for (int s2 = threadIdx.x; s2 < L; s2 += blockDim.x) lkeys[s2] = QM_EMPTY_KEY;
        for (int i = threadIdx.x; i < L * A.n_words; i += blockDim.x) lw[i] = A.init[i / L];
      }
      __syncthreads();
      for (uint64_t base = r0 + (uint64_t)warp * 32; base < r1; base += (uint64_t)warps * 32) {
        const uint64_t i = base + lane;
        const bool active = i < r1;
        uint64_t w[QM_MAX_VCOLS + 2];
        if (active) {
          const ulonglong2 *rec = reinterpret_cast<const ulonglong2 *>(ps.records + i * ps.rec_words);
#pragma unroll
          for (int k = 0; k < (QM_MAX_VCOLS + 2) / 2; ++k) {
            if (2 * k < 2 + QM_NV_BOUND(NV) && 2 * k < ps.rec_words) {
              const ulonglong2 v = __ldcs(rec + k);
              w[2 * k] = v.x;
              w[2 * k + 1] = v.y;
            } else {
              w[2 * k] = w[2 * k + 1] = 0;
            }
          }
        } else {
#pragma unroll
          for (int k = 0; k < QM_MAX_VCOLS + 2; ++k) w[k] = 0;
        }
        uint64_t vb[QM_MAX_VCOLS];
#pragma unroll
        for (int c = 0; c < QM_MAX_VCOLS; ++c) vb[c] = c < QM_NV_BOUND(NV) && c < nv ? w[2 + c] : 0;
        const int special = (int)((w[1] >> 32) & 0xff);
        const uint32_t vnull = (uint32_t)((w[1] >> 40) & 0xff);
        const uint64_t grow = (uint64_t)a.row_offset + (uint32_t)w[1];
        drain_apply<DD, NV, (NV > QM_MAX_VCOLS)>(P, lkeys, lw, L, &l_used, lane, active, w[0], special, grow, vb,
                                                vnull, scr);
      }
      __syncthreads();
      if (L > 0) {
        const int cw = A.w_count;
        for (int s2 = threadIdx.x; s2 < L; s2 += blockDim.x) {
          const uint64_t *lp = lw + s2;
          if (lp[(int64_t)cw * L] == 0) continue;
          if (!hashed && whole) {
            store_local(A, lp, L, P.table + (int64_t)s2 * P.stride + 1);
            continue;
          }
          const int64_t gs = hashed ? global_slot(P, lkeys[s2], 0) : s2;
          if (gs < 0) continue;
          merge_local(A, lp, L, P.table + gs * P.stride + 1);
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace qm

using namespace qm;

size_t qm_part_scan_smem(int parts) {
  return (size_t)(QM_SCAN_THREADS / 32) * QM_WQ * sizeof(uint32_t) + (size_t)(parts + 1) * sizeof(uint32_t);
}

size_t qm_part_agg_smem(int local_slots, int local_hash, int n_words) {
  return (size_t)local_slots * 8 * ((local_hash ? 1 : 0) + n_words) + (size_t)(QM_SCAN_THREADS / 32) * 64 * 8;
}

namespace {

// Kernel attributes and occupancy are set up once per instantiation (the
// largest shared memory any launch may ask for), not per launch.
constexpr size_t PART_SCAN_SMEM_MAX = (size_t)(QM_SCAN_THREADS / 32) * QM_WQ * 4 + (size_t)(8192 + 1) * 4;
constexpr size_t PART_AGG_SMEM_MAX = 200 * 1024;

template <auto Kernel>
cudaError_t set_smem_once(size_t bytes, int *per_sm_out = nullptr) {
  static std::once_flag once;  // one per kernel (the kernel is a template argument)
  const auto kernel = Kernel;
  static cudaError_t err = cudaSuccess;
  static int per_sm = 1;
  std::call_once(once, [&] {
    err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err == cudaSuccess)
      err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, QM_SCAN_THREADS, bytes);
  });
  if (per_sm_out) *per_sm_out = per_sm;
  return err;
}

template <int PASS, int NV, int KK>
cudaError_t part_scan_one(const qm_scan_args &a, const qm_part_spec &ps, cudaStream_t st) {
  const size_t smem = qm_part_scan_smem(ps.parts);
  cudaError_t e = set_smem_once<qm_part_scan<PASS, NV, KK>>(PART_SCAN_SMEM_MAX);
  if (e != cudaSuccess) return e;
  qm_part_scan<PASS, NV, KK><<<ps.blocks, QM_SCAN_THREADS, smem, st>>>(a, ps);
  return cudaGetLastError();
}

template <int PASS, int NV>
cudaError_t part_scan_kk(const qm_scan_args &a, const qm_part_spec &ps, int kk, cudaStream_t st) {
  if (kk == QM_KK_I64) return part_scan_one<PASS, NV, QM_KK_I64>(a, ps, st);
  if (kk == QM_KK_I32) return part_scan_one<PASS, NV, QM_KK_I32>(a, ps, st);
  return part_scan_one<PASS, NV, QM_KK_ANY>(a, ps, st);
}

template <int PASS>
cudaError_t part_scan_nv(const qm_scan_args &a, const qm_part_spec &ps, int kk, cudaStream_t st) {
  switch (a.agg.n_vcols) {
    case 1: return part_scan_kk<PASS, 1>(a, ps, kk, st);
    case 2: return part_scan_kk<PASS, 2>(a, ps, kk, st);
    default: return part_scan_kk<PASS, QM_NV_ANY>(a, ps, kk, st);
  }
}

int part_key_kind(const qm_keyspec &K) {
  if (K.n_cols == 1 && K.pack == QP_RAW && K.nulls[0] == nullptr) {
    if (K.dtype[0] == QM_I64) return QM_KK_I64;
    if (K.dtype[0] == QM_I32) return QM_KK_I32;
  }
  return QM_KK_ANY;
}

template <int DD, int NV>
cudaError_t part_agg_one(const qm_scan_args &a, const qm_part_spec &ps, int sm_count, cudaStream_t st) {
  const size_t smem = qm_part_agg_smem(ps.local_slots, ps.direct ? 0 : 1, a.agg.n_words);
  cudaError_t e = set_smem_once<qm_part_agg<DD, NV>>(PART_AGG_SMEM_MAX);
  if (e != cudaSuccess) return e;
  // two blocks of 16 warps per SM when their tables fit (register bound)
  const int per_sm = smem <= 100 * 1024 ? 2 : 1;
  const int blocks = sm_count * per_sm;
  // chunks: about 8 per block over the planned records, at least a few
  // table sizes each (the merge of a partition's table is paid per chunk)
  int64_t chunk = std::max<int64_t>(ps.rec_cap / ((int64_t)blocks * 8), (int64_t)ps.local_slots * 16);
  chunk = std::max<int64_t>(chunk, 8192);
  qm_part_agg<DD, NV><<<blocks, QM_SCAN_THREADS, smem, st>>>(a, ps, chunk);
  return cudaGetLastError();
}

}  // namespace

int qm_part_scan_blocks(int sm_count, int parts) {
  (void)parts;
  int per_sm = 1;
  if (set_smem_once<qm_part_scan<0, QM_NV_ANY, QM_KK_ANY>>(PART_SCAN_SMEM_MAX, &per_sm) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  return sm_count * std::min(std::max(per_sm, 1), 2);
}

cudaError_t qm_launch_part_scan(int pass, const qm_scan_args &a, const qm_part_spec &ps, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  const int kk = part_key_kind(a.key);
  return pass == 0 ? part_scan_nv<0>(a, ps, kk, st) : part_scan_nv<1>(a, ps, kk, st);
}

cudaError_t qm_launch_part_offsets(const qm_part_spec &ps, cudaStream_t st) {
  const int P1 = ps.parts + 1;
  const int blocks = (int)std::min<int64_t>(((int64_t)P1 * 32 + 255) / 256, 1024);
  qm_part_prefix<<<blocks, 256, 0, st>>>(ps);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  qm_part_bases<<<1, 1024, 0, st>>>(ps);
  return cudaGetLastError();
}

cudaError_t qm_launch_part_agg(const qm_scan_args &a, const qm_part_spec &ps, int sm_count, cudaStream_t st) {
  const bool fixed = [&] {
    for (int c = 0; c < a.agg.n_vcols; ++c)
      if (a.agg.vcol[c].flags & VF_FIXED) return true;
    return false;
  }();
  const int dd = a.dedupe != 0 ? 1 : 0;
  if (!fixed && a.agg.n_vcols == 1)
    return dd ? part_agg_one<1, 1>(a, ps, sm_count, st) : part_agg_one<0, 1>(a, ps, sm_count, st);
  if (!fixed && a.agg.n_vcols == 2)
    return dd ? part_agg_one<1, 2>(a, ps, sm_count, st) : part_agg_one<0, 2>(a, ps, sm_count, st);
  return dd ? part_agg_one<1, QM_NV_ANY>(a, ps, sm_count, st) : part_agg_one<0, QM_NV_ANY>(a, ps, sm_count, st);
}
