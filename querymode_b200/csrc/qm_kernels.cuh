// qm_kernels.cuh — device code of the fused filter -> GROUP BY path.
//
// One warp owns a tile of QM_TILE_ROWS consecutive rows (or selection
// entries).  Per tile:
//   1. predicates: each lane tests QM_R rows (lane, lane+32, ...), one term at
//      a time; a term's column is read only for rows still alive, so a
//      selective first term skips the sectors of later columns;
//   2. compaction: __ballot_sync masks + popcount prefix sums put the
//      surviving row offsets, in ascending row order, into a per-warp list;
//   3. aggregation: 32 survivors at a time, the lane gathers its row's key and
//      value cells, equal keys in the warp are merged with __match_any_sync
//      (one update per distinct key), and the leader updates the block-local
//      shared-memory table (or the global table when the key misses it).
// At block end the shared-memory table is merged into the global table with
// atomics.  Float sums are compensated (TwoSum of every atomic add: the old
// value returned by atomicAdd gives the exact rounding error, which goes to a
// second word), integer sums are exact 128-bit, MIN/MAX are integer atomics
// on an order-preserving image of the value.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/qm_gpu.h"
#include "qm_plan.h"

#define QM_FULL 0xffffffffu
#define QM_LOCAL_PROBE 8

namespace qm {

// murmur3 fmix64 finaliser — the hash the reference's LinearHashTable uses
// (wasm/src/query/vector_engine.zig:209-250)
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- column access ----------------------------------------------------------
// Column cells are read once per query: cache-streaming loads keep the group
// table (read-modify-written by atomics) resident in L2.
template <typename T>
__device__ __forceinline__ T ldcs(const void *p, int64_t r) {
  return __ldcs(reinterpret_cast<const T *>(p) + r);
}

__device__ __forceinline__ bool cell_null(const uint32_t *nb, int64_t r) {
  return nb != nullptr && ((__ldg(nb + (r >> 5)) >> (r & 31)) & 1u);
}

__device__ __forceinline__ int64_t ld_int(const void *p, int dtype, int64_t r) {
  return dtype == QM_I32 ? (int64_t)ldcs<int>(p, r) : (int64_t)ldcs<long long>(p, r);
}

__device__ __forceinline__ double ld_flt(const void *p, int dtype, int64_t r) {
  return dtype == QM_F32 ? (double)ldcs<float>(p, r) : ldcs<double>(p, r);
}

// order-preserving image of a double in int64 (after -0 -> +0)
__host__ __device__ __forceinline__ int64_t f2ord(double d) {
  int64_t b;
#ifdef __CUDA_ARCH__
  b = __double_as_longlong(d);
#else
  memcpy(&b, &d, 8);
#endif
  return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}

__host__ __device__ __forceinline__ double ord2f(int64_t o) {
  int64_t b = o >= 0 ? o : (o ^ 0x7fffffffffffffffLL);
#ifdef __CUDA_ARCH__
  return __longlong_as_double(b);
#else
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}

// ---- predicates -------------------------------------------------------------
__device__ __forceinline__ bool fcmp(double v, int op, double t) {
  switch (op) {
    case QC_EQ: return v == t;
    case QC_NEQ: return v != t;
    case QC_LT: return v < t;
    case QC_LTE: return v <= t;
    case QC_GT: return v > t;
    default: return v >= t;
  }
}

// JS: coerceCompare(number v, bigint b) -> BigInt(trunc(v)) <op> b, with a
// non-finite v compared as a number (src/decode.ts:480-485).
__device__ __forceinline__ bool fbig(double v, int op, int64_t b) {
  if (isnan(v)) return op == QC_NEQ;
  int c;
  if (isinf(v)) {
    c = v > 0 ? 1 : -1;
    if (op == QC_EQ) return false;
    if (op == QC_NEQ) return true;
  } else {
    double t = trunc(v);
    if (t >= 9223372036854775808.0) c = 1;
    else if (t < -9223372036854775808.0) c = -1;
    else {
      long long ti = (long long)t;
      c = ti < b ? -1 : (ti > b ? 1 : 0);
    }
  }
  switch (op) {
    case QC_EQ: return c == 0;
    case QC_NEQ: return c != 0;
    case QC_LT: return c < 0;
    case QC_LTE: return c <= 0;
    case QC_GT: return c > 0;
    default: return c >= 0;
  }
}

__device__ __forceinline__ bool fterm(const qm_term &t, double v) {
  switch (t.kind) {
    case QT_FRANGE:
      return ((t.op & 1) ? v >= t.f0 : v > t.f0) && ((t.op & 2) ? v <= t.f1 : v < t.f1);
    case QT_FCMP: return fcmp(v, t.op, t.f0);
    case QT_FBETWEEN: return v >= t.f0 && v <= t.f1;
    case QT_FNBETWEEN: return v < t.f0 || v > t.f1;
    default: return fbig(v, t.op, t.lo);
  }
}

// Tests term `t` on the lane's alive rows (bit j of m = row[j] alive).
template <typename ROWS>
__device__ __forceinline__ uint32_t eval_term(const qm_term &t, const ROWS &row, uint32_t m) {
  uint32_t pass = 0;
  if (t.kind <= QT_FALSE) {
    pass = t.kind == QT_TRUE ? ((1u << QM_R) - 1) : 0u;
  } else if (t.dtype == QM_I32 || t.dtype == QM_I64) {
    int64_t v[QM_R];
    if (t.dtype == QM_I32) {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) v[j] = ((m >> j) & 1) ? (int64_t)ldcs<int>(t.data, row(j)) : 0;
    } else {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) v[j] = ((m >> j) & 1) ? (int64_t)ldcs<long long>(t.data, row(j)) : 0;
    }
    const bool inr = t.kind == QT_IRANGE;
#pragma unroll
    for (int j = 0; j < QM_R; ++j) {
      bool in = v[j] >= t.lo && v[j] <= t.hi;
      pass |= (uint32_t)(in == inr) << j;
    }
  } else {
    double v[QM_R];
    if (t.dtype == QM_F32) {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) v[j] = ((m >> j) & 1) ? (double)ldcs<float>(t.data, row(j)) : 0.0;
    } else {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) v[j] = ((m >> j) & 1) ? ldcs<double>(t.data, row(j)) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < QM_R; ++j) pass |= (uint32_t)fterm(t, v[j]) << j;
  }
  if (t.nulls != nullptr) {
#pragma unroll
    for (int j = 0; j < QM_R; ++j)
      if (((m >> j) & 1) && cell_null(t.nulls, row(j)))
        pass = (pass & ~(1u << j)) | ((uint32_t)t.null_pass << j);
  }
  return m & pass;
}

// Full dense tile, lane owns rows e0 + 8*lane + j (j < 8): one or two
// 16-byte loads per column per lane, NULL bits as one byte per lane.
template <typename V, typename T, int PER>
__device__ __forceinline__ void load_contig(const void *data, int64_t r0, uint32_t m, T (&v)[QM_R]) {
  const V *p = reinterpret_cast<const V *>(reinterpret_cast<const T *>(data) + r0);
#pragma unroll
  for (int k = 0; k < QM_R / PER; ++k) {
    if ((m >> (k * PER)) & ((1u << PER) - 1)) {
      const V x = __ldcs(p + k);
      const T *xs = reinterpret_cast<const T *>(&x);
#pragma unroll
      for (int i = 0; i < PER; ++i) v[k * PER + i] = xs[i];
    } else {
#pragma unroll
      for (int i = 0; i < PER; ++i) v[k * PER + i] = T(0);
    }
  }
}

__device__ __forceinline__ uint32_t eval_term_contig(const qm_term &t, int64_t r0, uint32_t m) {
  uint32_t pass = 0;
  if (t.kind <= QT_FALSE) {
    pass = t.kind == QT_TRUE ? ((1u << QM_R) - 1) : 0u;
  } else if (t.dtype == QM_I32) {
    // the planner clamps int32 bounds to the int32 range: one unsigned
    // compare per cell tests lo <= v <= hi
    int w[QM_R];
    load_contig<int4, int, 4>(t.data, r0, m, w);
    const int lo = (int)t.lo;
    const uint32_t span = (uint32_t)((int)t.hi - lo);
#pragma unroll
    for (int j = 0; j < QM_R; ++j) pass |= (uint32_t)((uint32_t)(w[j] - lo) <= span) << j;
    if (t.kind == QT_INRANGE) pass = ~pass & ((1u << QM_R) - 1);
  } else if (t.dtype == QM_I64) {
    long long w[QM_R];
    load_contig<longlong2, long long, 2>(t.data, r0, m, w);
    const uint64_t span = (uint64_t)t.hi - (uint64_t)t.lo;
#pragma unroll
    for (int j = 0; j < QM_R; ++j) pass |= (uint32_t)((uint64_t)w[j] - (uint64_t)t.lo <= span) << j;
    if (t.kind == QT_INRANGE) pass = ~pass & ((1u << QM_R) - 1);
  } else {
    double v[QM_R];
    if (t.dtype == QM_F32) {
      float w[QM_R];
      load_contig<float4, float, 4>(t.data, r0, m, w);
#pragma unroll
      for (int j = 0; j < QM_R; ++j) v[j] = w[j];
    } else {
      load_contig<double2, double, 2>(t.data, r0, m, v);
    }
    if (t.kind == QT_FRANGE) {  // bounds are inclusive after planning
#pragma unroll
      for (int j = 0; j < QM_R; ++j) pass |= (uint32_t)(v[j] >= t.f0 && v[j] <= t.f1) << j;
    } else {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) pass |= (uint32_t)fterm(t, v[j]) << j;
    }
  }
  if (t.nulls != nullptr) {
    // r0 is a multiple of 8: the lane's 8 NULL bits are one byte
    const uint32_t nb = (__ldg(t.nulls + (r0 >> 5)) >> (r0 & 31)) & 0xffu;
    const uint32_t np = t.null_pass ? 0xffu : 0u;
    pass = (pass & ~nb) | (np & nb);
  }
  return m & pass;
}

// Pull a full tile of every filter column into L2 ahead of its evaluation
// (one 128-byte line per lane).
__device__ __forceinline__ void prefetch_tile_l2(const qm_pred &P, int64_t e0, int lane) {
  const int nt = P.n_groups > 0 ? P.group_end[P.n_groups - 1] : P.n_and;
  for (int i = 0; i < nt; ++i) {
    const qm_term &t = P.t[i];
    if (t.kind <= QT_FALSE) continue;
    const int elem = (t.dtype == QM_I32 || t.dtype == QM_F32) ? 4 : 8;
    if (lane < QM_TILE_ROWS * elem / 128) {
      const char *p = reinterpret_cast<const char *>(t.data) + e0 * elem + lane * 128;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }
}

__device__ __forceinline__ uint32_t eval_pred_contig(const qm_pred &P, int64_t r0, uint32_t m) {
  for (int i = 0; i < P.n_and; ++i) {
    if (!__any_sync(QM_FULL, m)) return 0;
    m = eval_term_contig(P.t[i], r0, m);
  }
  if (P.n_groups > 0) {
    uint32_t any = 0;
    int b = P.n_and;
    for (int g = 0; g < P.n_groups; ++g) {
      uint32_t mg = m & ~any;
      const int e = P.group_end[g];
      for (int i = b; i < e; ++i) {
        if (!__any_sync(QM_FULL, mg)) break;
        mg = eval_term_contig(P.t[i], r0, mg);
      }
      any |= mg;
      b = e;
    }
    m = any;
  }
  return m;
}

// ---- bulk async copies into shared memory (cp.async.bulk + mbarrier) ------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy; dst, src and bytes are multiples of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

#define QM_WAIT_LIMIT (1 << 22)

// Bounded wait for a phase of an mbarrier; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < QM_WAIT_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Term evaluation on a staged tile: rows e0 + j*32 + lane, cells read from
// the shared-memory copy (consecutive lanes, consecutive addresses).
__device__ __forceinline__ uint32_t eval_term_staged(const qm_term &t, const qm_staging &S, const uint8_t *buf,
                                                     int64_t e0, int lane, uint32_t m) {
  uint32_t pass = 0;
  if (t.kind <= QT_FALSE) {
    pass = t.kind == QT_TRUE ? ((1u << QM_R) - 1) : 0u;
  } else {
    const uint8_t *col = buf + S.off[t.sidx];
    if (t.dtype == QM_I32 || t.dtype == QM_I64) {
      const bool inr = t.kind == QT_IRANGE;
#pragma unroll
      for (int j = 0; j < QM_R; ++j) {
        const int64_t v = t.dtype == QM_I32 ? (int64_t)reinterpret_cast<const int *>(col)[j * 32 + lane]
                                            : (int64_t)reinterpret_cast<const long long *>(col)[j * 32 + lane];
        pass |= (uint32_t)((v >= t.lo && v <= t.hi) == inr) << j;
      }
    } else {
#pragma unroll
      for (int j = 0; j < QM_R; ++j) {
        const double v = t.dtype == QM_F32 ? (double)reinterpret_cast<const float *>(col)[j * 32 + lane]
                                           : reinterpret_cast<const double *>(col)[j * 32 + lane];
        pass |= (uint32_t)fterm(t, v) << j;
      }
    }
  }
  if (t.nulls != nullptr) {
#pragma unroll
    for (int j = 0; j < QM_R; ++j) {
      const uint32_t w = __ldg(t.nulls + ((e0 >> 5) + j));
      if ((w >> lane) & 1) pass = (pass & ~(1u << j)) | ((uint32_t)t.null_pass << j);
    }
  }
  return m & pass;
}

__device__ __forceinline__ uint32_t eval_pred_staged(const qm_pred &P, const qm_staging &S, const uint8_t *buf,
                                                     int64_t e0, int lane, uint32_t m) {
  for (int i = 0; i < P.n_and; ++i) {
    if (!__any_sync(QM_FULL, m)) return 0;
    m = eval_term_staged(P.t[i], S, buf, e0, lane, m);
  }
  if (P.n_groups > 0) {
    uint32_t any = 0;
    int b = P.n_and;
    for (int g = 0; g < P.n_groups; ++g) {
      uint32_t mg = m & ~any;
      const int e = P.group_end[g];
      for (int i = b; i < e; ++i) {
        if (!__any_sync(QM_FULL, mg)) break;
        mg = eval_term_staged(P.t[i], S, buf, e0, lane, mg);
      }
      any |= mg;
      b = e;
    }
    m = any;
  }
  return m;
}

// AND terms, then the OR of the groups' AND chains (src/decode.ts:558-578).
template <typename ROWS>
__device__ __forceinline__ uint32_t eval_pred(const qm_pred &P, const ROWS &row, uint32_t m) {
  for (int i = 0; i < P.n_and; ++i) {
    if (!__any_sync(QM_FULL, m)) return 0;
    m = eval_term(P.t[i], row, m);
  }
  if (P.n_groups > 0) {
    uint32_t any = 0;
    int b = P.n_and;
    for (int g = 0; g < P.n_groups; ++g) {
      uint32_t mg = m & ~any;
      const int e = P.group_end[g];
      for (int i = b; i < e; ++i) {
        if (!__any_sync(QM_FULL, mg)) break;
        mg = eval_term(P.t[i], row, mg);
      }
      any |= mg;
      b = e;
    }
    m = any;
  }
  return m;
}

// ---- group keys -------------------------------------------------------------
// Key word of one row.  special: 0 ordinary, 1 the key equals the empty-slot
// sentinel (hash mode), 2 NULL key.
// Key kinds a scan kernel can be specialised for (KK): 0 any plan; 1 one
// int64 column without NULLs; 2 one int32 column without NULLs; 3 no GROUP BY.
#define QM_KK_ANY 0
#define QM_KK_I64 1
#define QM_KK_I32 2
#define QM_KK_NONE 3
// Value-column counts (NV): 0..QM_MAX_VCOLS exactly, or QM_NV_ANY (read the
// plan's n_vcols at run time).
#define QM_NV_ANY (QM_MAX_VCOLS + 1)
#define QM_NV_BOUND(NV) ((NV) > QM_MAX_VCOLS ? QM_MAX_VCOLS : (NV))

// The payload columns of a tile (key columns, then value columns) into L2
// ahead of the survivors' gathers.
#ifndef QM_PREFETCH_PAYLOAD
#define QM_PREFETCH_PAYLOAD 0
#endif
template <int NV, int KK>
__device__ __forceinline__ void prefetch_payload_l2(const qm_keyspec &K, const qm_aggspec &A, int64_t e0, int lane) {
  auto line = [&](const void *data, int dtype) {
    const int elem = (dtype == QM_I32 || dtype == QM_F32) ? 4 : 8;
    if (lane < QM_TILE_ROWS * elem / 128) {
      const char *p = reinterpret_cast<const char *>(data) + e0 * elem + lane * 128;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  };
  if (KK == QM_KK_I64) line(K.data[0], QM_I64);
  else if (KK == QM_KK_I32) line(K.data[0], QM_I32);
  else if (KK != QM_KK_NONE)
    for (int i = 0; i < K.n_cols; ++i) line(K.data[i], K.dtype[i]);
  const int nv = NV > QM_MAX_VCOLS ? A.n_vcols : NV;
#pragma unroll
  for (int c = 0; c < QM_NV_BOUND(NV); ++c)
    if (c < nv) line(A.vcol[c].data, A.vcol[c].dtype);
}


template <int KK = QM_KK_ANY>
__device__ __forceinline__ uint64_t row_key(const qm_keyspec &K, int64_t r, int &special) {
  special = 0;
  if (KK == QM_KK_NONE) return 0;
  if (KK == QM_KK_I64 || KK == QM_KK_I32) {
    const uint64_t k = KK == QM_KK_I64 ? (uint64_t)ldcs<long long>(K.data[0], r)
                                       : (uint64_t)(int64_t)ldcs<int>(K.data[0], r);
    if (K.mode == QK_HASH && k == QM_EMPTY_KEY) special = 1;
    return k;
  }
  if (K.n_cols == 0) return 0;
  uint64_t k;
  if (K.pack == QP_CONCAT) {
    uint32_t a = (uint32_t)ldcs<int>(K.data[0], r), b = (uint32_t)ldcs<int>(K.data[1], r);
    k = ((uint64_t)a << 32) | b;
  } else if (K.pack == QP_DIGITS) {
    k = 0;
    for (int i = 0; i < K.n_cols; ++i) {
      uint64_t d;
      if (K.knullable[i] && cell_null(K.nulls[i], r)) d = 0;
      else d = (uint64_t)(ld_int(K.data[i], K.dtype[i], r) - K.kbase[i]) + (uint64_t)K.knullable[i];
      k += d * K.kmul[i];
    }
  } else {
    if (cell_null(K.nulls[0], r)) {
      special = 2;
      return 0;
    }
    switch (K.dtype[0]) {
      case QM_I32: k = (uint64_t)(int64_t)ldcs<int>(K.data[0], r); break;
      case QM_I64: k = (uint64_t)ldcs<long long>(K.data[0], r); break;
      default: {
        // String(v) identity: -0 and 0 share "0", every NaN is "NaN"
        double d = ld_flt(K.data[0], K.dtype[0], r);
        if (d == 0.0) d = 0.0;
        k = isnan(d) ? 0x7ff8000000000000ULL : (uint64_t)__double_as_longlong(d);
      }
    }
  }
  if (K.mode == QK_HASH && k == QM_EMPTY_KEY) special = 1;
  return k;
}

__device__ __forceinline__ void set_error(qm_status *st, int code) {
  atomicCAS(&st->error, 0, code);
}

// Linear probing with a CAS claim of the key word.  Accumulator words are
// pre-initialised, so a claimed slot is immediately usable.
__device__ __forceinline__ int64_t global_find(uint64_t *table, int stride, int log2cap,
                                               uint64_t key, int max_probe, qm_status *st) {
  const uint64_t mask = (1ULL << log2cap) - 1;
  uint64_t s = fmix64(key) & mask;
  for (int p = 0; p < max_probe; ++p) {
    unsigned long long *kp = reinterpret_cast<unsigned long long *>(table + s * stride);
    uint64_t k = *reinterpret_cast<volatile unsigned long long *>(kp);
    if (k == key) return (int64_t)s;
    if (k == QM_EMPTY_KEY) {
      uint64_t prev = atomicCAS(kp, QM_EMPTY_KEY, key);
      if (prev == QM_EMPTY_KEY) {
        atomicAdd(&st->groups_inserted, 1ULL);
        return (int64_t)s;
      }
      if (prev == key) return (int64_t)s;
    }
    s = (s + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ int64_t global_slot(const qm_scan_args &a, uint64_t key, int special) {
  if (a.key.mode == QK_NONE) return 0;
  if (a.key.mode == QK_DIRECT) {
    if (special == 2) return a.n_slots;
    uint64_t d = key - (uint64_t)a.key.base;
    if (d >= (uint64_t)a.n_slots) {
      set_error(a.status, QM_DEV_RANGE);
      return -1;
    }
    return (int64_t)d;
  }
  if (special) return a.n_slots + special - 1;
  int64_t s = global_find(a.table, a.stride, a.log2cap, key, a.max_probe, a.status);
  if (s < 0) set_error(a.status, QM_DEV_OVERFLOW);
  return s;
}

// A group's slot from its key, without inserting (the key is in the table).
__device__ __forceinline__ int64_t find_slot(const qm_scan_args &a, uint64_t key, int special) {
  if (a.key.mode == QK_NONE) return 0;
  if (a.key.mode == QK_DIRECT) {
    if (special == 2) return a.n_slots;
    const uint64_t d = key - (uint64_t)a.key.base;
    return d < (uint64_t)a.n_slots ? (int64_t)d : -1;
  }
  if (special) return a.n_slots + special - 1;
  const uint64_t mask = (1ULL << a.log2cap) - 1;
  uint64_t s = fmix64(key) & mask;
  for (int p = 0; p < a.max_probe; ++p) {
    const uint64_t k = a.table[s * a.stride];
    if (k == key) return (int64_t)s;
    if (k == QM_EMPTY_KEY) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}

// Block-local lookup.  New keys are admitted only while the table is at
// most half full (`used` counts admissions), so a miss meets an empty slot
// within a few probes and goes to the global table.
__device__ __forceinline__ int local_find(uint64_t *lkeys, int L, uint64_t key, int *used) {
  uint32_t s = (uint32_t)fmix64(key) & (uint32_t)(L - 1);
  for (int p = 0; p < QM_LOCAL_PROBE; ++p) {
    uint64_t k = reinterpret_cast<volatile uint64_t *>(lkeys)[s];
    if (k == key) return (int)s;
    if (k == QM_EMPTY_KEY) {
      if (*reinterpret_cast<volatile int *>(used) >= (L >> 1)) return -1;
      uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long *>(lkeys + s), QM_EMPTY_KEY, key);
      if (prev == QM_EMPTY_KEY) {
        atomicAdd(used, 1);
        return (int)s;
      }
      if (prev == key) return (int)s;
    }
    s = (s + 1) & (uint32_t)(L - 1);
  }
  return -1;
}

// ---- accumulator updates ------------------------------------------------------
__device__ __forceinline__ void add128(uint64_t *lo, uint64_t *hi, uint64_t vlo, int64_t vhi) {
  if (vlo != 0) {
    uint64_t old = atomicAdd(reinterpret_cast<unsigned long long *>(lo), (unsigned long long)vlo);
    if (old + vlo < old) vhi += 1;
  }
  if (vhi != 0) atomicAdd(reinterpret_cast<unsigned long long *>(hi), (unsigned long long)vhi);
}

// Compensated atomic add: atomicAdd returns the old value, so the rounding
// error of old + x is recovered exactly (TwoSum) and added, with the
// contribution's own low part xc, to the low word.
__device__ __forceinline__ void fsum_add(uint64_t *hp, uint64_t *lp, double x, double xc) {
  if (x == 0.0 && xc == 0.0) return;
  double old = atomicAdd(reinterpret_cast<double *>(hp), x);
  double s = old + x;
  if (!isfinite(s)) return;
  double bb = s - old;
  double err = (old - (s - bb)) + (x - bb);
  double add = xc + err;
  if (add != 0.0) atomicAdd(reinterpret_cast<double *>(lp), add);
}

// Split summation: x = xh + xl exactly; the high words only ever hold
// multiples of ulp(split) below split in magnitude, so their atomic adds are
// exact in any order and need no returned value.  Non-finite x goes to the
// high word as it is (Infinity / NaN propagate as in the reference's sum).
__device__ __forceinline__ void split_parts(double x, double split, double &xh, double &xl) {
  if (!isfinite(x)) {
    xh = x;
    xl = 0.0;
    return;
  }
  xh = __dsub_rn(__dadd_rn(x, split), split);
  xl = __dsub_rn(x, xh);
}

__device__ __forceinline__ void split_add(uint64_t *hp, uint64_t *lp, double x, double split) {
  double xh, xl;
  split_parts(x, split, xh, xl);
  if (xh != 0.0 || isnan(xh)) atomicAdd(reinterpret_cast<double *>(hp), xh);
  if (xl != 0.0) atomicAdd(reinterpret_cast<double *>(lp), xl);
}

__device__ __forceinline__ void two_sum_acc(double &s, double &c, double x) {
  double t = s + x;
  if (isfinite(t)) {
    double bb = t - s;
    c += (s - (t - bb)) + (x - bb);
  }
  s = t;
}

// ---- fixed-point float sums (VF_FIXED) -------------------------------------
// A finite x as round(x / 2^fxe) (ties to even), a 128-bit two's-complement
// integer.  Planning keeps |x| < 2^(fxe + 126), so the value fits; sums of
// these integers are exact and do not depend on the order of the adds.
__device__ __forceinline__ void fx_parts(double x, int fxe, uint64_t &lo, int64_t &hi) {
  const uint64_t b = (uint64_t)__double_as_longlong(x);
  const int ex = (int)((b >> 52) & 0x7ff);
  uint64_t m = b & ((1ULL << 52) - 1);
  int e2 = -1074;  // zero or subnormal: m * 2^-1074
  if (ex != 0) {
    m |= 1ULL << 52;
    e2 = ex - 1075;
  }
  const int sh = e2 - fxe;  // x = m * 2^sh units
  unsigned __int128 v = 0;
  if (m != 0) {
    if (sh >= 0) {
      v = (unsigned __int128)m << sh;
    } else if (sh > -64) {
      const int r = -sh;
      uint64_t q = m >> r;
      const uint64_t rem = m & ((1ULL << r) - 1), half = 1ULL << (r - 1);
      if (rem > half || (rem == half && (q & 1))) q++;
      v = q;
    }
  }
  if (b >> 63) v = (unsigned __int128)0 - v;
  lo = (uint64_t)v;
  hi = (int64_t)(uint64_t)(v >> 64);
}

// One cell of a fixed-point SUM column: its integer value, or its
// non-finite bit (NaN 1, +Infinity 2, -Infinity 4); `stale` when the cell is
// beyond the planned range.
__device__ __forceinline__ void fx_cell(const qm_vcol &vc, double x, uint64_t &lo, int64_t &hi, uint32_t &nf,
                                        bool &stale) {
  lo = 0;
  hi = 0;
  nf = 0;
  if (isnan(x)) {
    nf = 1;
  } else if (isinf(x)) {
    nf = x > 0 ? 2u : 4u;
  } else if (fabs(x) >= vc.fx_max) {
    stale = true;
  } else {
    fx_parts(x, vc.fx_exp, lo, hi);
  }
}

// A fixed-point sum's value: NaN if a NaN or both infinities were seen, else
// the infinity seen, else the integer scaled back (rounded once, to nearest).
__device__ __forceinline__ double i128_to_f64(uint64_t lo, int64_t hi);
__device__ __forceinline__ double fx_value(uint64_t lo, int64_t hi, uint64_t nf, int fxe) {
  if ((nf & 1) || (nf & 6) == 6) return __longlong_as_double(0x7ff8000000000000LL);
  if (nf & 2) return __longlong_as_double(0x7ff0000000000000LL);
  if (nf & 4) return __longlong_as_double((long long)0xfff0000000000000ULL);
  return ldexp(i128_to_f64(lo, hi), fxe);
}

__device__ __forceinline__ uint64_t pick(const uint64_t (&v)[QM_MAX_VCOLS], int i) {
  uint64_t r = 0;
#pragma unroll
  for (int c = 0; c < QM_MAX_VCOLS; ++c)
    if (c == i) r = v[c];
  return r;
}

// Value cell c of a row: a plain register when the kernel knows the column
// count (c is then a compile-time index), else a select over the array.
template <int NV>
__device__ __forceinline__ uint64_t vget(const uint64_t (&vb)[QM_MAX_VCOLS], int c) {
  if constexpr (NV > QM_MAX_VCOLS) return pick(vb, c);
  else return vb[c];
}

// Monotone updates: the word only ever decreases (min) or increases (max),
// so a plain read that already beats the value makes the atomic redundant.
__device__ __forceinline__ void min_u64(uint64_t *p, uint64_t v) {
  if (v < *reinterpret_cast<volatile uint64_t *>(p)) atomicMin(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
}
__device__ __forceinline__ void min_i64(uint64_t *p, int64_t v) {
  if (v < (int64_t)*reinterpret_cast<volatile uint64_t *>(p)) atomicMin(reinterpret_cast<long long *>(p), (long long)v);
}
__device__ __forceinline__ void max_i64(uint64_t *p, int64_t v) {
  if (v > (int64_t)*reinterpret_cast<volatile uint64_t *>(p)) atomicMax(reinterpret_cast<long long *>(p), (long long)v);
}
// In the global table the read test costs an L2 round trip that the warp
// waits for; there the atomics go out unconditionally (no returned value, so
// they are fire-and-forget reductions).
__device__ __forceinline__ void upd_min_u64(uint64_t *p, uint64_t v, bool local) {
  if (local) min_u64(p, v);
  else atomicMin(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
}
__device__ __forceinline__ void upd_min_i64(uint64_t *p, int64_t v, bool local) {
  if (local) min_i64(p, v);
  else atomicMin(reinterpret_cast<long long *>(p), (long long)v);
}
__device__ __forceinline__ void upd_max_i64(uint64_t *p, int64_t v, bool local) {
  if (local) max_i64(p, v);
  else atomicMax(reinterpret_cast<long long *>(p), (long long)v);
}

// Accumulator word updates, atomic or (plain = the slot is private to the
// calling lane's warp and only one lane writes it) a plain read-modify-write.
__device__ __forceinline__ void acc_add_u64(uint64_t *p, uint64_t v, bool plain) {
  if (plain) *p += v;
  else atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
}
__device__ __forceinline__ void acc_add_f64(uint64_t *p, double v, bool plain) {
  if (plain) *reinterpret_cast<double *>(p) += v;
  else atomicAdd(reinterpret_cast<double *>(p), v);
}
__device__ __forceinline__ void acc_min_u64(uint64_t *p, uint64_t v, bool plain, bool local) {
  if (plain) *p = min(*p, v);
  else upd_min_u64(p, v, local);
}
__device__ __forceinline__ void acc_min_i64(uint64_t *p, int64_t v, bool plain) {
  if (plain) *p = (uint64_t)min((int64_t)*p, v);
  else atomicMin(reinterpret_cast<long long *>(p), (long long)v);
}
__device__ __forceinline__ void acc_max_i64(uint64_t *p, int64_t v, bool plain) {
  if (plain) *p = (uint64_t)max((int64_t)*p, v);
  else atomicMax(reinterpret_cast<long long *>(p), (long long)v);
}
__device__ __forceinline__ void acc_add128(uint64_t *lo, uint64_t *hi, uint64_t vlo, int64_t vhi, bool plain) {
  if (!plain) {
    add128(lo, hi, vlo, vhi);
    return;
  }
  const uint64_t o = *lo, n = o + vlo;
  *lo = n;
  *hi = (uint64_t)((int64_t)*hi + vhi + (n < o ? 1 : 0));
}
__device__ __forceinline__ void acc_fsum(uint64_t *hp, uint64_t *lp, double x, double xc, bool plain) {
  if (!plain) {
    fsum_add(hp, lp, x, xc);
    return;
  }
  if (x == 0.0 && xc == 0.0) return;
  const double old = __longlong_as_double((long long)*hp);
  const double s = old + x;
  *hp = (uint64_t)__double_as_longlong(s);
  if (!isfinite(s)) return;
  const double bb = s - old;
  const double add = xc + ((old - (s - bb)) + (x - bb));
  if (add != 0.0) *reinterpret_cast<double *>(lp) += add;
}

// Butterfly reductions over all 32 lanes (every lane gets the result): the
// peer loops below are O(peers), this is O(log 32) for the common case of a
// whole warp in one group (no GROUP BY, or a dominant key).
template <class T, class OP>
__device__ __forceinline__ T warp_allreduce(T v, OP op) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = op(v, __shfl_xor_sync(QM_FULL, v, o));
  return v;
}

// Reduction of `v` over the calling lane's peer group, for every lane of
// `act` (the lanes executing this; peers is a subset of act).  One loop of
// `iters` steps (the largest group's size - 1) runs in lockstep for all
// groups, so groups do not serialise on divergent loops; a whole-warp group
// takes the butterfly.
template <class T, class OP>
__device__ __forceinline__ T group_reduce(T v, unsigned act, unsigned peers, int lane, int iters, OP op) {
  if (peers == QM_FULL) return warp_allreduce(v, op);
  T r = v;
  unsigned rem = peers & ~(1u << lane);
  for (int it = 0; it < iters; ++it) {
    const int src = rem ? __ffs(rem) - 1 : lane;
    const T x = __shfl_sync(act, v, src);
    if (rem) {
      r = op(r, x);
      rem &= rem - 1;
    }
  }
  return r;
}

// Apply one compacted row (merged with its equal-key peers) to a slot whose
// accumulator word w lives at tp[w * ws].  Every lane of `act` executes this
// (the shuffles need them); only group leaders, with tp != nullptr, write.
// iters = (largest peer group in act) - 1.
// FX: the kernel carries the fixed-point (VF_FIXED) sum paths; kernels
// specialised for a column count and key kind leave them out (their plans
// never use them, and the extra paths cost the hot loop instructions).
template <bool FX = true>
__device__ __forceinline__ void apply_row(const qm_aggspec &A, uint64_t *tp, int ws, bool local, unsigned act,
                                          unsigned peers, int iters, int lane, uint64_t grow,
                                          const uint64_t (&vb)[QM_MAX_VCOLS], uint32_t vnull, bool plain = false,
                                          qm_status *st = nullptr) {
  const bool full = peers == QM_FULL;
  auto umin = [](uint64_t x, uint64_t y) { return min(x, y); };
  auto imin = [](int64_t x, int64_t y) { return min(x, y); };
  auto imax = [](int64_t x, int64_t y) { return max(x, y); };
  auto iadd = [](int64_t x, int64_t y) { return x + y; };
  auto fadd = [](double x, double y) { return x + y; };
  for (int i = 0; i < A.n_accs; ++i) {
    const qm_acc ac = A.acc[i];
    uint64_t *w0 = tp ? tp + (int64_t)ac.word * ws : nullptr;
    uint64_t *w1 = tp ? tp + (int64_t)(ac.word + 1) * ws : nullptr;
    if (ac.kind == QA_COUNT) {
      if (tp) acc_add_u64(w0, (uint64_t)__popc(peers), plain);
      continue;
    }
    if (ac.kind == QA_FIRST) {
      const uint64_t first = iters > 0 ? group_reduce(grow, act, peers, lane, iters, umin) : grow;
      if (tp) acc_min_u64(w0, first, plain, local);
      continue;
    }
    const bool valid = !((vnull >> ac.vcol) & 1);
    const uint64_t raw = pick(vb, ac.vcol);
    switch (ac.kind) {
      case QA_NN: {
        const unsigned nn = __popc(__ballot_sync(act, valid) & peers);
        if (tp && nn) acc_add_u64(w0, (uint64_t)nn, plain);
        break;
      }
      case QA_ISUM: {
        const int64_t v = valid ? (int64_t)raw : 0;
        if (!ac.wide) {
          const int64_t s = iters > 0 ? group_reduce(v, act, peers, lane, iters, iadd) : v;
          if (tp && s != 0) {
            if (local || ac.narrow) acc_add_u64(w0, (uint64_t)s, plain);
            else add128(w0, w1, (uint64_t)s, s < 0 ? -1 : 0);
          }
        } else {
          // 128-bit sum of up to 32 int64 cells
          uint64_t lo = (uint64_t)v;
          int64_t hi = v < 0 ? -1 : 0;
          if (full) {
#pragma unroll
            for (int o = 16; o; o >>= 1) {
              const uint64_t xl = __shfl_xor_sync(QM_FULL, lo, o);
              const int64_t xh = __shfl_xor_sync(QM_FULL, hi, o);
              const uint64_t nlo = lo + xl;
              hi += xh + (nlo < lo ? 1 : 0);
              lo = nlo;
            }
          } else {
            unsigned rem = peers & ~(1u << lane);
            for (int it = 0; it < iters; ++it) {
              const int src = rem ? __ffs(rem) - 1 : lane;
              const int64_t x = __shfl_sync(act, v, src);
              if (rem) {
                const uint64_t nlo = lo + (uint64_t)x;
                hi += (x < 0 ? -1 : 0) + (nlo < lo ? 1 : 0);
                lo = nlo;
                rem &= rem - 1;
              }
            }
          }
          if (tp && (lo != 0 || hi != 0)) acc_add128(w0, w1, lo, hi, plain);
        }
        break;
      }
      case QA_FSUM: {
        const double v = valid ? __longlong_as_double((long long)raw) : 0.0;
        const qm_vcol &fv = A.vcol[ac.vcol];
        if (FX && (fv.flags & VF_FIXED)) {
          uint64_t lo;
          int64_t hi;
          uint32_t nf;
          bool stale = false;
          fx_cell(fv, v, lo, hi, nf, stale);
          if (stale && st) set_error(st, QM_DEV_STALE);
          if (full) {
            nf = warp_allreduce(nf, [](uint32_t x, uint32_t y) { return x | y; });
#pragma unroll
            for (int o = 16; o; o >>= 1) {
              const uint64_t xl = __shfl_xor_sync(QM_FULL, lo, o);
              const int64_t xh = __shfl_xor_sync(QM_FULL, hi, o);
              const uint64_t nlo = lo + xl;
              hi += xh + (nlo < lo ? 1 : 0);
              lo = nlo;
            }
          } else {
            const uint64_t lo0 = lo;
            const int64_t hi0 = hi;
            const uint32_t nf0 = nf;
            unsigned rem = peers & ~(1u << lane);
            for (int it = 0; it < iters; ++it) {
              const int src = rem ? __ffs(rem) - 1 : lane;
              const uint64_t xl = __shfl_sync(act, lo0, src);
              const int64_t xh = __shfl_sync(act, hi0, src);
              const uint32_t xn = __shfl_sync(act, nf0, src);
              if (rem) {
                const uint64_t nlo = lo + xl;
                hi += xh + (nlo < lo ? 1 : 0);
                lo = nlo;
                nf |= xn;
                rem &= rem - 1;
              }
            }
          }
          if (tp) {
            if (lo != 0 || hi != 0) acc_add128(w0, w1, lo, hi, plain);
            if (nf) {
              uint64_t *wn = tp + (int64_t)fv.w_nf * ws;
              if (plain) *wn |= nf;
              else atomicOr(reinterpret_cast<unsigned long long *>(wn), (unsigned long long)nf);
            }
          }
          break;
        }
        const double split = fv.split;
        if (split != 0.0) {
          double h, l;
          split_parts(v, split, h, l);
          if (iters > 0) {
            h = group_reduce(h, act, peers, lane, iters, fadd);  // exact: multiples of ulp(split) below split
            l = group_reduce(l, act, peers, lane, iters, fadd);
          }
          if (tp) {
            if (h != 0.0 || isnan(h)) acc_add_f64(w0, h, plain);
            if (l != 0.0) acc_add_f64(w1, l, plain);
          }
          break;
        }
        double s = v, c = 0.0;
        if (full) {
#pragma unroll
          for (int o = 16; o; o >>= 1) {
            const double xs = __shfl_xor_sync(QM_FULL, s, o);
            const double xc = __shfl_xor_sync(QM_FULL, c, o);
            double cc = c + xc;
            two_sum_acc(s, cc, xs);
            c = cc;
          }
        } else {
          unsigned rem = peers & ~(1u << lane);
          for (int it = 0; it < iters; ++it) {
            const int src = rem ? __ffs(rem) - 1 : lane;
            const double x = __shfl_sync(act, v, src);
            if (rem) {
              two_sum_acc(s, c, x);
              rem &= rem - 1;
            }
          }
        }
        if (tp) acc_fsum(w0, w1, s, c, plain);
        break;
      }
      case QA_IMIN:
      case QA_IMAX: {
        const bool mx = ac.kind == QA_IMAX;
        int64_t v = valid ? (int64_t)raw : (mx ? INT64_MIN : INT64_MAX);
        if (iters > 0) v = mx ? group_reduce(v, act, peers, lane, iters, imax) : group_reduce(v, act, peers, lane, iters, imin);
        if (tp && v != (mx ? INT64_MIN : INT64_MAX)) {
          if (mx) acc_max_i64(w0, v, plain);
          else acc_min_i64(w0, v, plain);
        }
        break;
      }
      case QA_FMIN:
      case QA_FMAX: {
        const bool mx = ac.kind == QA_FMAX;
        const double d = __longlong_as_double((long long)raw);
        const bool ok = valid && !isnan(d);  // NaN never wins '<' / '>' (src/partial-agg.ts:80-81)
        int64_t o = ok ? f2ord(d == 0.0 ? 0.0 : d) : (mx ? INT64_MIN : INT64_MAX);
        if (iters > 0) o = mx ? group_reduce(o, act, peers, lane, iters, imax) : group_reduce(o, act, peers, lane, iters, imin);
        if (tp && o != (mx ? INT64_MIN : INT64_MAX)) {
          if (mx) acc_max_i64(w0, o, plain);
          else acc_min_i64(w0, o, plain);
        }
        break;
      }
      case QA_FZERO: {
        const double d = __longlong_as_double((long long)raw);
        const bool z = valid && d == 0.0;
        uint64_t code = z ? ((grow << 1) | (raw >> 63)) : ~0ULL;
        if (__any_sync(act, z) && iters > 0) code = group_reduce(code, act, peers, lane, iters, umin);
        if (tp && code != ~0ULL) acc_min_u64(w0, code, plain, false);
        break;
      }
    }
  }
}

// One row's update of the slot whose word w lives at tp[w * ws]: straight
// line per value column, values already gathered into vb (NULL bits in
// vnull) so the cell loads overlap the key lookup.
#ifndef QM_GLOBAL_READ_TEST
#define QM_GLOBAL_READ_TEST 0
#endif
template <int NV = QM_NV_ANY, bool FX = true>
__device__ __forceinline__ void agg_row(const qm_aggspec &A, uint64_t *tp, int ws, bool local,
                                        uint64_t grow, const uint64_t (&vb)[QM_MAX_VCOLS], uint32_t vnull,
                                        qm_status *st = nullptr) {
  // In the global table, the FIRST word and the MIN / MAX words of the first
  // two value columns are read up front, in one L2 round trip; the atomics
  // then go out only where the row beats the word read.  A word only moves
  // one way, so a stale read can cause an unneeded atomic, never skip one.
  uint64_t g_first = 0;
  int64_t g_mn[2] = {0, 0}, g_mx[2] = {0, 0};
  const bool gtest = QM_GLOBAL_READ_TEST && !local;
  if (gtest) {
    if (A.w_first >= 0) g_first = __ldcg(reinterpret_cast<const unsigned long long *>(tp + (int64_t)A.w_first * ws));
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (c >= A.n_vcols) break;
      const int f = A.vcol[c].flags;
      if (f & VF_MIN) g_mn[c] = __ldcg(reinterpret_cast<const long long *>(tp + (int64_t)A.vcol[c].w_min * ws));
      if (f & VF_MAX) g_mx[c] = __ldcg(reinterpret_cast<const long long *>(tp + (int64_t)A.vcol[c].w_max * ws));
    }
  }
  atomicAdd(reinterpret_cast<unsigned long long *>(tp + (int64_t)A.w_count * ws), 1ULL);
  if (A.w_first >= 0) {
    uint64_t *p = tp + (int64_t)A.w_first * ws;
    if (!gtest) upd_min_u64(p, grow, local);
    else if (grow < g_first) atomicMin(reinterpret_cast<unsigned long long *>(p), (unsigned long long)grow);
  }
  auto gmin = [&](int c, uint64_t *p, int64_t v) {
    if (gtest && c < 2) {
      if (v < g_mn[c]) atomicMin(reinterpret_cast<long long *>(p), (long long)v);
    } else {
      upd_min_i64(p, v, local);
    }
  };
  auto gmax = [&](int c, uint64_t *p, int64_t v) {
    if (gtest && c < 2) {
      if (v > g_mx[c]) atomicMax(reinterpret_cast<long long *>(p), (long long)v);
    } else {
      upd_max_i64(p, v, local);
    }
  };
#pragma unroll
  for (int c = 0; c < QM_NV_BOUND(NV); ++c) {
    if (NV > QM_MAX_VCOLS && c >= A.n_vcols) break;
    if ((vnull >> c) & 1) continue;
    const qm_vcol &vc = A.vcol[c];
    const int f = vc.flags;
    if (f & VF_NN) atomicAdd(reinterpret_cast<unsigned long long *>(tp + (int64_t)vc.w_nn * ws), 1ULL);
    if (vc.dtype == QM_I32 || vc.dtype == QM_I64) {
      const int64_t v = (int64_t)vb[c];
      if ((f & VF_SUM) && v != 0) {
        uint64_t *w0 = tp + (int64_t)vc.w_sum * ws;
        if ((local && !(f & VF_WIDE)) || (f & VF_NARROW))
          atomicAdd(reinterpret_cast<unsigned long long *>(w0), (unsigned long long)v);
        else add128(w0, w0 + ws, (uint64_t)v, v < 0 ? -1 : 0);
      }
      if (f & VF_MIN) gmin(c, tp + (int64_t)vc.w_min * ws, v);
      if (f & VF_MAX) gmax(c, tp + (int64_t)vc.w_max * ws, v);
    } else {
      const double d = __longlong_as_double((long long)vb[c]);
      if (f & VF_SUM) {
        uint64_t *w0 = tp + (int64_t)vc.w_sum * ws;
        if (FX && (f & VF_FIXED)) {
          uint64_t lo;
          int64_t hi;
          uint32_t nf;
          bool stale = false;
          fx_cell(vc, d, lo, hi, nf, stale);
          if (stale && st) set_error(st, QM_DEV_STALE);
          if (lo != 0 || hi != 0) add128(w0, w0 + ws, lo, hi);
          if (nf) atomicOr(reinterpret_cast<unsigned long long *>(tp + (int64_t)vc.w_nf * ws), (unsigned long long)nf);
        } else if (vc.split != 0.0) {
          split_add(w0, w0 + ws, d, vc.split);
        } else {
          fsum_add(w0, w0 + ws, d, 0.0);
        }
      }
      if ((f & (VF_MIN | VF_MAX)) && !isnan(d)) {  // NaN never wins '<' / '>'
        const int64_t o = f2ord(d == 0.0 ? 0.0 : d);
        if (f & VF_MIN) gmin(c, tp + (int64_t)vc.w_min * ws, o);
        if (f & VF_MAX) gmax(c, tp + (int64_t)vc.w_max * ws, o);
      }
      if ((f & VF_ZERO) && d == 0.0) upd_min_u64(tp + (int64_t)vc.w_zero * ws, (grow << 1) | (vb[c] >> 63), local);
    }
  }
}

// Equal-slot merge for a drain round: lanes in `peers` (same block-local
// slot, mask `lmask` = every lane taking this path) sum their additive
// contributions through the warp's shared scratch, and the group leader adds
// them once; MIN / MAX / FIRST stay per lane (64-bit min/max atomics resolve
// conflicts in hardware, and most are skipped by the read test).
template <int NV = QM_NV_ANY, bool FX = true>
__device__ __forceinline__ void agg_row_merged(const qm_aggspec &A, uint64_t *tp, int L, unsigned lmask, unsigned peers,
                                               int lane, uint64_t grow, const uint64_t (&vb)[QM_MAX_VCOLS],
                                               uint32_t vnull, uint64_t *scr, qm_status *st = nullptr) {
  const bool leader = lane == __ffs(peers) - 1;
  if (leader) atomicAdd(reinterpret_cast<unsigned long long *>(tp + (int64_t)A.w_count * L), (unsigned long long)__popc(peers));
  if (A.w_first >= 0) min_u64(tp + (int64_t)A.w_first * L, grow);
  const int nv = NV > QM_MAX_VCOLS ? A.n_vcols : NV;
#pragma unroll
  for (int c = 0; c < nv; ++c) {
    const qm_vcol &vc = A.vcol[c];
    const int f = vc.flags;
    const bool valid = !((vnull >> c) & 1);
    if (f & VF_NN) {
      const unsigned nn = __popc(__ballot_sync(lmask, valid) & peers);
      if (leader && nn) atomicAdd(reinterpret_cast<unsigned long long *>(tp + (int64_t)vc.w_nn * L), (unsigned long long)nn);
    }
    const bool isint = vc.dtype == QM_I32 || vc.dtype == QM_I64;
    const uint64_t raw = vget<NV>(vb, c);
    if (f & VF_SUM) {
      uint64_t *w0 = tp + (int64_t)vc.w_sum * L;
      if (isint) {
        scr[lane] = valid ? raw : 0;
        __syncwarp(lmask);
        if (leader) {
          // 128-bit sum of up to 32 cells (int64 cells can carry out of 64 bits)
          uint64_t lo = 0;
          int64_t hi = 0;
          for (unsigned m = peers; m; m &= m - 1) {
            const int64_t x = (int64_t)scr[__ffs(m) - 1];
            const uint64_t nlo = lo + (uint64_t)x;
            hi += (x < 0 ? -1 : 0) + (nlo < lo ? 1 : 0);
            lo = nlo;
          }
          if (f & VF_WIDE) {
            if (lo != 0 || hi != 0) add128(w0, w0 + L, lo, hi);
          } else if (lo != 0) {
            atomicAdd(reinterpret_cast<unsigned long long *>(w0), (unsigned long long)lo);  // int32 cells: fits
          }
        }
        __syncwarp(lmask);
      } else if (FX && (f & VF_FIXED)) {
        const double d = valid ? __longlong_as_double((long long)raw) : 0.0;
        uint64_t lo;
        int64_t hi;
        uint32_t nf;
        bool stale = false;
        fx_cell(vc, d, lo, hi, nf, stale);
        if (stale && st) set_error(st, QM_DEV_STALE);
        if (nf) atomicOr(reinterpret_cast<unsigned long long *>(tp + (int64_t)vc.w_nf * L), (unsigned long long)nf);
        scr[lane] = lo;
        scr[32 + lane] = (uint64_t)hi;
        __syncwarp(lmask);
        if (leader) {
          uint64_t slo = 0;
          int64_t shi = 0;
          for (unsigned m = peers; m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            const uint64_t nlo = slo + scr[src];
            shi += (int64_t)scr[32 + src] + (nlo < slo ? 1 : 0);
            slo = nlo;
          }
          if (slo != 0 || shi != 0) add128(w0, w0 + L, slo, shi);
        }
        __syncwarp(lmask);
      } else {
        const double d = valid ? __longlong_as_double((long long)raw) : 0.0;
        double h, l;
        if (vc.split != 0.0) split_parts(d, vc.split, h, l);
        else {
          h = d;
          l = 0.0;
        }
        scr[lane] = (uint64_t)__double_as_longlong(h);
        scr[32 + lane] = (uint64_t)__double_as_longlong(l);
        __syncwarp(lmask);
        if (leader) {
          if (vc.split != 0.0) {
            double sh = 0.0, sl = 0.0;
            for (unsigned m = peers; m; m &= m - 1) {
              const int src = __ffs(m) - 1;
              sh += __longlong_as_double((long long)scr[src]);  // exact: grid multiples below split
              sl += __longlong_as_double((long long)scr[32 + src]);
            }
            if (sh != 0.0) atomicAdd(reinterpret_cast<double *>(w0), sh);
            if (sl != 0.0) atomicAdd(reinterpret_cast<double *>(w0 + L), sl);
          } else {
            double s = 0.0, cc = 0.0;
            for (unsigned m = peers; m; m &= m - 1) two_sum_acc(s, cc, __longlong_as_double((long long)scr[__ffs(m) - 1]));
            fsum_add(w0, w0 + L, s, cc);
          }
        }
        __syncwarp(lmask);
      }
    }
    if (!valid) continue;
    if (isint) {
      const int64_t v = (int64_t)raw;
      if (f & VF_MIN) min_i64(tp + (int64_t)vc.w_min * L, v);
      if (f & VF_MAX) max_i64(tp + (int64_t)vc.w_max * L, v);
    } else {
      const double d = __longlong_as_double((long long)raw);
      if ((f & (VF_MIN | VF_MAX)) && !isnan(d)) {
        const int64_t o = f2ord(d == 0.0 ? 0.0 : d);
        if (f & VF_MIN) min_i64(tp + (int64_t)vc.w_min * L, o);
        if (f & VF_MAX) max_i64(tp + (int64_t)vc.w_max * L, o);
      }
      if ((f & VF_ZERO) && d == 0.0) min_u64(tp + (int64_t)vc.w_zero * L, (grow << 1) | (raw >> 63));
    }
  }
}

// Gather a row's value cells (float32 widened to double, as JS numbers).
template <int NV = QM_NV_ANY>
__device__ __forceinline__ void gather_values(const qm_aggspec &A, int64_t row, uint64_t (&vb)[QM_MAX_VCOLS],
                                              uint32_t &vnull) {
  vnull = 0;
#pragma unroll
  for (int c = 0; c < QM_MAX_VCOLS; ++c) {
    vb[c] = 0;
    if (c < QM_NV_BOUND(NV) && (NV <= QM_MAX_VCOLS || c < A.n_vcols)) {
      const qm_vcol &vc = A.vcol[c];
      if (cell_null(vc.nulls, row)) vnull |= 1u << c;
      else if (vc.dtype == QM_I32 || vc.dtype == QM_I64) vb[c] = (uint64_t)ld_int(vc.data, vc.dtype, row);
      else vb[c] = (uint64_t)__double_as_longlong(ld_flt(vc.data, vc.dtype, row));
    }
  }
}

// Merge one block-local slot (words at lp[w * L]) into global slot words gp.
__device__ __forceinline__ void merge_local(const qm_aggspec &A, const uint64_t *lp, int L, uint64_t *gp) {
  for (int i = 0; i < A.n_accs; ++i) {
    const qm_acc ac = A.acc[i];
    const uint64_t v0 = lp[(int64_t)ac.word * L];
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
        if (ac.wide) add128(g0, g1, v0, (int64_t)lp[(int64_t)(ac.word + 1) * L]);
        else if (v0 && ac.narrow) atomicAdd(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
        else if (v0) add128(g0, g1, v0, (int64_t)v0 < 0 ? -1 : 0);
        break;
      case QA_FNF:
        if (v0) atomicOr(reinterpret_cast<unsigned long long *>(g0), (unsigned long long)v0);
        break;
      case QA_FSUM:
        if (A.vcol[ac.vcol].flags & VF_FIXED) {
          const uint64_t v1 = lp[(int64_t)(ac.word + 1) * L];
          if (v0 || v1) add128(g0, g1, v0, (int64_t)v1);
        } else if (A.vcol[ac.vcol].split != 0.0) {
          const double h = __longlong_as_double((long long)v0);
          const double l = __longlong_as_double((long long)lp[(int64_t)(ac.word + 1) * L]);
          if (h != 0.0 || isnan(h)) atomicAdd(reinterpret_cast<double *>(g0), h);
          if (l != 0.0) atomicAdd(reinterpret_cast<double *>(g1), l);
        } else {
          fsum_add(g0, g1, __longlong_as_double((long long)v0),
                   __longlong_as_double((long long)lp[(int64_t)(ac.word + 1) * L]));
        }
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

// Fold block-local slot words src[w * L] into dst[w * L] (both in this
// block's shared memory, no other writer): the per-warp copies of a private
// table collapse into one before the global merge.
__device__ __forceinline__ void merge_plain(const qm_aggspec &A, uint64_t *dst, const uint64_t *src, int L) {
  for (int i = 0; i < A.n_accs; ++i) {
    const qm_acc ac = A.acc[i];
    const int64_t w0 = (int64_t)ac.word * L, w1 = (int64_t)(ac.word + 1) * L;
    switch (ac.kind) {
      case QA_COUNT:
      case QA_NN: dst[w0] += src[w0]; break;
      case QA_FIRST:
      case QA_FZERO: dst[w0] = min(dst[w0], src[w0]); break;
      case QA_ISUM:
        if (ac.wide) acc_add128(dst + w0, dst + w1, src[w0], (int64_t)src[w1], true);
        else dst[w0] += src[w0];
        break;
      case QA_FNF: dst[w0] |= src[w0]; break;
      case QA_FSUM:
        if (A.vcol[ac.vcol].flags & VF_FIXED) {
          acc_add128(dst + w0, dst + w1, src[w0], (int64_t)src[w1], true);
        } else if (A.vcol[ac.vcol].split != 0.0) {
          acc_add_f64(dst + w0, __longlong_as_double((long long)src[w0]), true);
          acc_add_f64(dst + w1, __longlong_as_double((long long)src[w1]), true);
        } else {
          acc_fsum(dst + w0, dst + w1, __longlong_as_double((long long)src[w0]),
                   __longlong_as_double((long long)src[w1]), true);
        }
        break;
      case QA_IMIN:
      case QA_FMIN: acc_min_i64(dst + w0, (int64_t)src[w0], true); break;
      case QA_IMAX:
      case QA_FMAX: acc_max_i64(dst + w0, (int64_t)src[w0], true); break;
    }
  }
}

// Applies one survivor per lane (key word, special flag, global row and
// gathered cells; lanes with active = false sit out) to the block-local
// table or else the global table.
template <int DD = 2, int NV = QM_NV_ANY, bool FX = true>
__device__ __forceinline__ void drain_apply(const qm_scan_args &a, uint64_t *lkeys, uint64_t *lw, int L, int *l_used,
                                            int lane, bool active, uint64_t key, int special, uint64_t grow,
                                            const uint64_t (&vb)[QM_MAX_VCOLS], uint32_t vnull, uint64_t *scr) {
  const qm_aggspec &A = a.agg;
  if (DD == 2 ? a.dedupe != 0 : DD == 1) {
    const unsigned act = __ballot_sync(QM_FULL, active);
    if (!active) return;
    unsigned peers = __match_any_sync(act, key);
    if (__any_sync(act, special != 0)) peers &= __match_any_sync(act, special);
    const bool leader = lane == __ffs(peers) - 1;
    uint64_t *tp = nullptr;
    int ws = 1;
    bool local = false;
    if (leader) {
      int ls = -1;
      if (L > 0) {
        if (!a.local_hash) ls = (int)global_slot(a, key, special);
        else if (special == 0) ls = local_find(lkeys, L, key, l_used);
      }
      if (ls >= 0) {
        tp = lw + ls;
        ws = L;
        local = true;
      } else if (!(L > 0 && !a.local_hash)) {
        const int64_t gs = global_slot(a, key, special);
        if (gs >= 0) tp = a.table + gs * a.stride + 1;
      }
    }
    const int iters = (int)__reduce_max_sync(act, (unsigned)__popc(peers)) - 1;
    apply_row<FX>(A, tp, ws, local, act, peers, iters, lane, grow, vb, vnull, local && a.priv, FX ? a.status : nullptr);
    return;
  }
  int ls = -1;
  if (active && L > 0) {
    if (!a.local_hash) ls = (int)global_slot(a, key, special);
    else if (special == 0) ls = local_find(lkeys, L, key, l_used);
  }
  const bool loc = active && ls >= 0;
  const unsigned lmask = __ballot_sync(QM_FULL, loc);
  unsigned peers = 0;
  if (loc) peers = __match_any_sync(lmask, ls);
  const bool merge = __any_sync(QM_FULL, (peers & (peers - 1)) != 0);
  if (loc) {
    if (merge) agg_row_merged<NV, FX>(A, lw + ls, L, lmask, peers, lane, grow, vb, vnull, scr, FX ? a.status : nullptr);
    else agg_row<NV, FX>(A, lw + ls, L, true, grow, vb, vnull, FX ? a.status : nullptr);
  } else if (active && !(L > 0 && !a.local_hash)) {
    const int64_t gs = global_slot(a, key, special);
    if (gs >= 0) agg_row<NV, FX>(A, a.table + gs * a.stride + 1, 1, false, grow, vb, vnull, FX ? a.status : nullptr);
  }
}

// Aggregates one survivor per lane (lanes with active = false sit out):
// gathers its key and value cells, then drain_apply.
// DD: 0 / 1 = the plan's dedupe flag fixed at compile time (separate kernels
// keep each path's registers and code apart), 2 = read it from the plan.
template <int DD = 2, int NV = QM_NV_ANY, int KK = QM_KK_ANY, bool FX = true>
__device__ __forceinline__ void drain_round_any(const qm_scan_args &a, uint64_t *lkeys, uint64_t *lw, int L,
                                                int *l_used, int lane, bool active, int64_t row, uint64_t *scr) {
  uint64_t grow = 0, key = 0;
  int special = 0;
  uint64_t vb[QM_MAX_VCOLS];
  uint32_t vnull = 0;
  if (active) {
    grow = (uint64_t)(a.row_offset + row);
    key = row_key<KK>(a.key, row, special);
    gather_values<NV>(a.agg, row, vb, vnull);
  }
  drain_apply<DD, NV, FX>(a, lkeys, lw, L, l_used, lane, active, key, special, grow, vb, vnull, scr);
}


// Number(bigint): round to nearest, ties to even.
__device__ __forceinline__ double i128_to_f64(uint64_t lo, int64_t hi) {
  const bool neg = hi < 0;
  if (neg) {  // negate the 128-bit value
    lo = ~lo + 1;
    hi = ~hi + (lo == 0 ? 1 : 0);
  }
  const uint64_t uhi = (uint64_t)hi;
  double r;
  if (uhi == 0) {
    r = __ull2double_rn(lo);
  } else {
    const int shift = 64 - __clzll((long long)uhi);  // drop `shift` bits
    const uint64_t top = (uhi << (64 - shift)) | (lo >> shift);
    const bool sticky = (lo << (64 - shift)) != 0;
    uint64_t keep = top >> 11;
    const uint64_t rem = top & 0x7ff;
    const bool guard = (rem >> 10) & 1;
    const bool st = sticky || (rem & 0x3ff);
    if (guard && (st || (keep & 1))) keep++;
    r = ldexp((double)keep, shift + 11);
  }
  return neg ? -r : r;
}

__device__ __forceinline__ void set_null(unsigned char *out, int64_t null_offset, int64_t i) {
  atomicOr(reinterpret_cast<unsigned *>(out + null_offset) + (i >> 5), 1u << (i & 31));
}

// Finalize slot `s` of a group table into output row `i` (keys, then each
// aggregate; NULL bits in the output's word bitmaps).
// BYTES: NULL flags go to one byte per output row at nullbytes + nboff[k]
// (every nullable output writes 0 or 1, so no clearing is needed);
// otherwise set bits in the word bitmap at out + null_offset.
// A NULL output cell: its flag, and zero in the data cell (the output
// buffer is not cleared beforehand).
__device__ __forceinline__ void zero_cell(unsigned char *col, int dtype, int64_t i) {
  if (dtype == QM_I32 || dtype == QM_F32) {
    reinterpret_cast<uint32_t *>(col)[i] = 0;
  } else if (dtype == QM_I128) {
    reinterpret_cast<uint64_t *>(col)[2 * i] = 0;
    reinterpret_cast<uint64_t *>(col)[2 * i + 1] = 0;
  } else {
    reinterpret_cast<uint64_t *>(col)[i] = 0;
  }
}
#define NULL_OUT()                                  \
  do {                                              \
    if (BYTES) nullbytes[nboff[k] + i] = 1;         \
    else set_null(out, o.null_offset, i);           \
    zero_cell(col, o.dtype, i);                     \
  } while (0)
template <bool BYTES>
__device__ __forceinline__ void emit_group(const uint64_t *t, int stride, uint64_t s, int64_t i, const qm_keyspec &K,
                                           int64_t n_slots, const qm_outspec &O, unsigned char *out,
                                           unsigned char *nullbytes, const int64_t *nboff) {
  const uint64_t *w = t + s * stride + 1;
  // reconstruct the key word
  bool knull = false;
  uint64_t key = 0;
  if (K.mode == QK_DIRECT) {
    if ((int64_t)s == n_slots) knull = true;
    else key = (uint64_t)K.base + s;
  } else if (K.mode == QK_HASH) {
    if ((int64_t)s == n_slots) key = QM_EMPTY_KEY;
    else if ((int64_t)s == n_slots + 1) knull = true;
    else key = t[s * stride];
  }
  for (int k = 0; k < O.n_out; ++k) {
    const qm_out &o = O.o[k];
    unsigned char *col = out + o.offset;
    if (BYTES && nboff[k] >= 0) nullbytes[nboff[k] + i] = 0;
    if (o.kind == QO_KEY) {
      if (knull) {
        NULL_OUT();
        continue;
      }
      if (K.pack == QP_CONCAT) {
        reinterpret_cast<int32_t *>(col)[i] = (int32_t)(o.src == 0 ? (key >> 32) : key);
      } else if (K.pack == QP_DIGITS) {
        const int c = o.src;
        const uint64_t d = (key / K.kmul[c]) % K.kradix[c];
        if (K.knullable[c] && d == 0) {
          NULL_OUT();
          continue;
        }
        const int64_t v = K.kbase[c] + (int64_t)(d - (uint64_t)K.knullable[c]);
        if (o.dtype == QM_I32) reinterpret_cast<int32_t *>(col)[i] = (int32_t)v;
        else reinterpret_cast<int64_t *>(col)[i] = v;
      } else if (o.dtype == QM_I32) {
        reinterpret_cast<int32_t *>(col)[i] = (int32_t)(int64_t)key;
      } else {
        reinterpret_cast<uint64_t *>(col)[i] = key;
      }
      continue;
    }
    if (o.kind == QO_COUNT) {
      reinterpret_cast<int64_t *>(col)[i] = (int64_t)w[o.word];
      continue;
    }
    const uint64_t nn = w[o.nn_word];
    if (nn == 0) {
      NULL_OUT();
      continue;
    }
    switch (o.kind) {
      case QO_SUM_F:
      case QO_AVG_F: {
        double s2 = o.fixed ? fx_value(w[o.word], (int64_t)w[o.word + 1], w[o.nf_word], o.fx_exp)
                            : __longlong_as_double((long long)w[o.word]) + __longlong_as_double((long long)w[o.word + 1]);
        reinterpret_cast<double *>(col)[i] = o.kind == QO_SUM_F ? s2 : s2 / (double)nn;
        break;
      }
      case QO_SUM_I2F:
      case QO_AVG_I2F: {
        const int64_t hi = o.narrow ? ((int64_t)w[o.word] >> 63) : (int64_t)w[o.word + 1];
        double s2 = i128_to_f64(w[o.word], hi);
        reinterpret_cast<double *>(col)[i] = o.kind == QO_SUM_I2F ? s2 : s2 / (double)nn;
        break;
      }
      case QO_SUM_I128:
        reinterpret_cast<uint64_t *>(col)[2 * i] = w[o.word];
        reinterpret_cast<uint64_t *>(col)[2 * i + 1] = w[o.word + 1];
        break;
      case QO_AVG_BIG: {
        // bigAvg(bigSum, 0, count): Number(sum / n) + Number(sum % n) / n
        const __int128 sum = (__int128)(((unsigned __int128)(uint64_t)w[o.word + 1] << 64) | w[o.word]);
        const __int128 q = sum / (__int128)nn, r = sum % (__int128)nn;
        const double qd = i128_to_f64((uint64_t)q, (int64_t)(q >> 64));
        const double rd = i128_to_f64((uint64_t)r, (int64_t)(r >> 64));
        reinterpret_cast<double *>(col)[i] = qd + (rd + 0.0) / (double)nn;
        break;
      }
      case QO_MIN_I:
      case QO_MAX_I:
        if (o.dtype == QM_I32) reinterpret_cast<int32_t *>(col)[i] = (int32_t)(int64_t)w[o.word];
        else reinterpret_cast<int64_t *>(col)[i] = (int64_t)w[o.word];
        break;
      case QO_MIN_F:
      case QO_MAX_F: {
        const int64_t ov = (int64_t)w[o.word];
        double d = ord2f(ov);
        // a zero result takes the sign of the first zero seen (strict
        // '<' / '>' keep the first of -0 and 0, src/partial-agg.ts:80-81)
        if (ov == 0 && o.zero_word >= 0 && w[o.zero_word] != ~0ULL && (w[o.zero_word] & 1)) d = -0.0;
        reinterpret_cast<double *>(col)[i] = d;
        break;
      }
    }
  }
}

#undef NULL_OUT

__device__ __forceinline__ void emit_group_bytes(const uint64_t *t, int stride, uint64_t s, int64_t i,
                                                 const qm_keyspec &K, int64_t n_slots, const qm_outspec &O,
                                                 unsigned char *out, unsigned char *nullbytes, const int64_t *nboff) {
  emit_group<true>(t, stride, s, i, K, n_slots, O, out, nullbytes, nboff);
}

}  // namespace qm
