// qm_api.cu — the C ABI of include/qm_gpu.h: contexts, HBM-resident tables,
// the planner that lowers a query, execution, finalize, results.
//
// The planner folds the reference's JS comparison coercions into the kernel's
// bounds:
//   * int64 column vs number t: coerceCompare turns t into BigInt(trunc(t))
//     (src/decode.ts:480-485), so the test is an exact integer comparison
//     with trunc(t);
//   * int32 / float column vs number: plain JS number comparison — exact for
//     int32 cells, IEEE for float cells (NaN compares false, != is true);
//   * bigint t: exact integer comparison (int columns) or
//     BigInt(trunc(v)) <op> t (float columns).
// Every integer test becomes one inclusive range or its complement, clamped
// to the column type; empty / full ranges become constants.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <map>
#include <mutex>
#include <string>
#include <deque>
#include <functional>
#include <vector>

#include "../../include/qm_gpu.h"
#include "qm_launch.h"
#include "qm_plan.h"

typedef __int128 i128;

namespace {

// ------------------------------------------------------------ device buffers
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct HostBuf {
  void *p = nullptr;
  size_t bytes = 0;
  bool carved = false;  // part of a pinned slab (returns to the pool, never freed alone)
};

// Pinned host buffers handed to results and recycled when they are
// destroyed (shared by the context and its results, which may outlive it).
struct PinnedPool {
  std::mutex mu;
  std::vector<HostBuf> free;
  std::vector<void *> slabs;                      // page-locked slabs buffers are carved from
  std::vector<std::pair<char *, size_t>> space;   // the slabs' uncarved ends
  ~PinnedPool() {
    for (auto &b : free)
      if (!b.carved) cudaFreeHost(b.p);
    for (void *s : slabs) cudaFreeHost(s);
  }
  // Buffers are power-of-two sized (results of similar size share them) and
  // kept up to a byte cap: allocating or freeing pinned memory costs far
  // more than a query (page-locking takes about 0.4 ms per MB and holds up
  // every other thread's CUDA calls meanwhile; freeing synchronises the
  // device).  Buffers up to CARVE_MAX are carved from SLAB-sized page-locked
  // slabs, so new results cost one page-locking per slab, not one per
  // buffer; carved buffers stay in the pool.
  static constexpr size_t CACHE_CAP = (size_t)16 << 30;
  static constexpr size_t MAX_BUFFERS = 4096;
  static constexpr size_t SLAB = (size_t)512 << 20;
  static constexpr size_t CARVE_MAX = (size_t)64 << 20;
  static size_t class_of(size_t bytes) {
    size_t want = 64 * 1024;
    while (want < bytes) want <<= 1;
    return want;
  }
  // under mu: a new slab (false when page-locking fails)
  bool add_slab() {
    void *sp = nullptr;
    if (cudaMallocHost(&sp, SLAB) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    slabs.push_back(sp);
    space.emplace_back(static_cast<char *>(sp), SLAB);
    return true;
  }
  // Page-lock slabs for at least `bytes` of buffers ahead of need (a server
  // does this at creation, so its first requests pay no page-locking).
  void reserve(size_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    size_t have = 0;
    for (auto &sp : space) have += sp.second;
    while (have < bytes && add_slab()) have += SLAB;
  }
  bool acquire(size_t bytes, HostBuf &out) {
    const size_t want = class_of(bytes);
    {
      // the smallest free buffer of at least the request's class, at most
      // twice it (a large buffer is not spent on a small result)
      std::lock_guard<std::mutex> lk(mu);
      int best = -1;
      for (int i = 0; i < (int)free.size(); i++)
        if (free[i].bytes >= want && free[i].bytes <= 2 * want && (best < 0 || free[i].bytes < free[best].bytes))
          best = i;
      if (best >= 0) {
        out = free[best];
        free.erase(free.begin() + best);
        return true;
      }
      if (want <= CARVE_MAX) {
        int at = -1;
        for (int i = 0; i < (int)space.size() && at < 0; i++)
          if (space[i].second >= want) at = i;
        if (at < 0 && add_slab()) at = (int)space.size() - 1;
        if (at >= 0) {
          out.p = space[at].first;
          out.bytes = want;
          out.carved = true;
          space[at].first += want;
          space[at].second -= want;
          return true;
        }
      }
    }
    if (cudaMallocHost(&out.p, want) != cudaSuccess) {
      cudaGetLastError();
      out = HostBuf();
      return false;
    }
    out.bytes = want;
    out.carved = false;
    return true;
  }
  // Kept for reuse up to the caps; beyond them the smallest buffers of their
  // own go first (the large ones cost the most to page-lock again).
  void release(HostBuf &b) {
    if (!b.p) return;
    std::vector<void *> drop;
    {
      std::lock_guard<std::mutex> lk(mu);
      free.push_back(b);
      size_t cached = 0, own = 0;
      for (auto &f : free)
        if (!f.carved) {
          cached += f.bytes;
          own++;
        }
      while ((cached > CACHE_CAP || own > MAX_BUFFERS) && own > 0) {
        int s = -1;
        for (int i = 0; i < (int)free.size(); i++)
          if (!free[i].carved && (s < 0 || free[i].bytes < free[s].bytes)) s = i;
        cached -= free[s].bytes;
        own--;
        drop.push_back(free[s].p);
        free.erase(free.begin() + s);
      }
    }
    for (void *p : drop) cudaFreeHost(p);
    b = HostBuf();
  }
};

// Device blocks of destroyed tables' columns, kept (up to a cap) for the
// next table's columns of about the same size: tables created and dropped
// per host batch or per ingest then cost no cudaMalloc / cudaFree (and
// cudaFree synchronises the device).  Emptied whenever an allocation fails.
struct DevPool {
  std::mutex mu;
  std::vector<std::pair<void *, size_t>> free;
  size_t cached = 0;
  static size_t round(size_t b) {
    return (std::max<size_t>(b, 256) + ((size_t)1 << 21) - 1) & ~(((size_t)1 << 21) - 1);
  }
  void *take(size_t bytes, size_t &got) {
    std::lock_guard<std::mutex> lk(mu);
    const size_t want = round(bytes);
    int best = -1;
    for (int i = 0; i < (int)free.size(); i++)
      if (free[i].second >= want && free[i].second <= want + want / 4 &&
          (best < 0 || free[i].second < free[best].second))
        best = i;
    if (best < 0) return nullptr;
    void *p = free[best].first;
    got = free[best].second;
    cached -= got;
    free.erase(free.begin() + best);
    return p;
  }
  bool keep(void *p, size_t bytes, size_t cap) {
    std::lock_guard<std::mutex> lk(mu);
    if (cached + bytes > cap || free.size() >= 256) return false;
    free.push_back({p, bytes});
    cached += bytes;
    return true;
  }
  bool trim() {
    std::lock_guard<std::mutex> lk(mu);
    const bool any = !free.empty();
    for (auto &f : free) cudaFree(f.first);
    free.clear();
    cached = 0;
    return any;
  }
};

}  // namespace

// Chunks of a large result emitted and copied to host memory in turn.
#ifndef QM_EMIT_CHUNKS
#define QM_EMIT_CHUNKS 8
#endif

struct qm_ctx {
  int device = 0;
  int sm_count = 0;
  int64_t hbm_bytes = 0;
  cudaStream_t stream = nullptr;      // where work is ordered
  cudaStream_t own_stream = nullptr;  // the context's own stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evs0 = nullptr, evs1 = nullptr;
  int launches = 0;  // kernels of this library launched since the last reset
  qm_tuning tuning{0, -1, 0, 0, 0, 0};  // local_slots, dedupe, blocks_per_sm, stage_depth, partitioned
  std::string err;
  // grow-only scratch reused across runs of this context
  DevBuf table, status, keys, slots, keys2, slots2, sort_temp, counter, out, hll;
  DevBuf masks, counts, offsets, sel_out, sel_in;
  DevBuf agg_spare;  // group table of a destroyed qm_agg, reused by the next one
  DevBuf fbits, fcounts, franks;  // first-row bitmap, its popcounts and prefix sums
  DevBuf perm;                    // slot of each ranked output row (large results)
  DevBuf zstat, zones;           // zone-map statistics pass; the kept zones of a query
  DevBuf part_counts, part_offsets, part_bases, part_records;  // partitioned aggregation
  // post-aggregate ORDER BY / LIMIT: sort keys, row orders, scratch, result
  DevBuf post_last, post_hi, post_lo, post_idx, post_idx2, post_k1, post_k2, post_l1, post_l2, post_temp, out2;
  std::vector<DevBuf> staged;  // per-column uploads of pushed host batches
  HostBuf hout, hstatus;
  std::shared_ptr<PinnedPool> pool = std::make_shared<PinnedPool>();
  DevPool dpool;  // column blocks of destroyed tables
  // side stream for the statistics of columns being uploaded
  cudaStream_t aux = nullptr;
  cudaEvent_t aux_ev = nullptr;
  // chunked copies of a large result while its later chunks are emitted
  cudaStream_t copy = nullptr;
  cudaEvent_t copy_ev[QM_EMIT_CHUNKS + 1] = {};
  DevBuf wbounds;
  DevBuf ustat;
};

namespace {

int set_err(qm_ctx *ctx, int code, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return set_err(ctx, QM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int ensure(qm_ctx *ctx, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return QM_OK;
  const size_t old_bytes = b.p ? b.bytes : 0;
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  // grow by at least half again (and to a 2 MiB multiple), so buffers that
  // track a changing working set are reallocated rarely: cudaFree
  // synchronises the device
  size_t want = std::max<size_t>(bytes, 256);
  if (old_bytes) want = std::max(want, old_bytes + old_bytes / 2);
  if (want > ((size_t)1 << 21)) want = (want + ((size_t)1 << 21) - 1) & ~(((size_t)1 << 21) - 1);
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (ctx->dpool.trim()) e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      b.p = nullptr;
      return set_err(ctx, QM_ERR_OOM, "cudaMalloc(%zu): %s", want, cudaGetErrorString(e));
    }
  }
  b.bytes = want;
  return QM_OK;
}

// ensure() for buffers used on one stream only: grown with stream-ordered
// allocation (cudaFreeAsync / cudaMallocAsync on that stream), so growing
// one batch's buffers does not synchronise the device under the other
// batches in flight (a serving lane growing to a larger request).
int ensure_on(qm_ctx *ctx, DevBuf &b, size_t bytes, cudaStream_t st) {
  if (b.bytes >= bytes && b.p) return QM_OK;
  const size_t old_bytes = b.p ? b.bytes : 0;
  if (b.p) {
    cudaFreeAsync(b.p, st);
    b.p = nullptr;
    b.bytes = 0;
  }
  size_t want = std::max<size_t>(bytes, 256);
  if (old_bytes) want = std::max(want, old_bytes + old_bytes / 2);
  if (want > ((size_t)1 << 21)) want = (want + ((size_t)1 << 21) - 1) & ~(((size_t)1 << 21) - 1);
  cudaError_t e = cudaMallocAsync(&b.p, want, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return set_err(ctx, QM_ERR_OOM, "cudaMallocAsync(%zu): %s", want, cudaGetErrorString(e));
  }
  b.bytes = want;
  return QM_OK;
}

int ensure_host(qm_ctx *ctx, HostBuf &b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return QM_OK;
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.bytes = 0;
  size_t want = std::max<size_t>(bytes, 4096);
  cudaError_t e = cudaMallocHost(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, QM_ERR_OOM, "cudaMallocHost(%zu): %s", want, cudaGetErrorString(e));
  }
  b.bytes = want;
  return QM_OK;
}

void release(DevBuf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

int64_t qm_f2ord_host(double d) {
  int64_t b;
  memcpy(&b, &d, 8);
  return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}

size_t dtype_size(int d) { return d == QM_I32 || d == QM_F32 ? 4 : (d == QM_I128 ? 16 : 8); }
bool is_int(int d) { return d == QM_I32 || d == QM_I64; }
bool valid_dtype(int d) { return d == QM_I32 || d == QM_I64 || d == QM_F32 || d == QM_F64; }

// ------------------------------------------------------------ columns
struct DevCol {
  std::string name;
  int dtype = QM_F64;
  void *data = nullptr;
  uint32_t *nulls = nullptr;
  bool own_data = false, own_nulls = false;
  size_t data_block = 0, nulls_block = 0;  // pooled block sizes (0: plain cudaMalloc)
  bool has_minmax = false;
  long long mn = 0, mx = 0;
  bool has_hll = false;
  double hll = 0;
  bool has_maxabs = false;
  double maxabs = 0;  // max |x| over finite non-NULL cells (float columns)
  bool has_zones = false;  // zone maps (QM_ZONE_ROWS rows per zone)
  std::vector<int64_t> zmin, zmax, zcount;  // float columns: double bits
};

}  // namespace

struct qm_table {
  qm_ctx *ctx = nullptr;
  int64_t n_rows = 0;
  std::vector<DevCol> cols;
  // sampled bounds on the rows a predicate selects, by the predicate's bytes
  // (planning estimates: a stale one only costs a regrowth)
  std::unordered_map<uint64_t, int64_t> sel_bounds;
};

namespace {

// Device memory for a table column: a pooled block of about its size, else
// a new 2 MiB-rounded one (the pool is emptied and the allocation retried
// when the device is full).  `block` receives the block's size.
void *col_alloc(qm_ctx *ctx, size_t bytes, size_t &block) {
  void *p = ctx->dpool.take(bytes, block);
  if (p) return p;
  block = DevPool::round(bytes);
  if (cudaMalloc(&p, block) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    if (ctx->dpool.trim() && cudaMalloc(&p, block) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
  }
  return p;
}

// Blocks kept for reuse: at most an eighth of the device's memory.
void col_release(qm_ctx *ctx, void *p, size_t block) {
  if (!p) return;
  if (!ctx || !block || !ctx->dpool.keep(p, block, (size_t)ctx->hbm_bytes / 8)) cudaFree(p);
}

void free_col(qm_ctx *ctx, DevCol &c) {
  if (c.own_data && c.data) col_release(ctx, c.data, c.data_block);
  if (c.own_nulls && c.nulls) col_release(ctx, c.nulls, c.nulls_block);
  c.data = nullptr;
  c.nulls = nullptr;
}

// Copy a QMCB-style byte bitmap into a 32-bit-word device bitmap.
int upload_nulls(qm_ctx *ctx, const uint8_t *host_bits, int64_t n, uint32_t **out, size_t &block) {
  size_t words = (size_t)((n + 31) / 32) + 1;
  uint32_t *d = (uint32_t *)col_alloc(ctx, words * 4, block);
  if (!d) return set_err(ctx, QM_ERR_OOM, "null bitmap alloc (%zu bytes)", words * 4);
  *out = d;
  CK(cudaMemsetAsync(d, 0, words * 4, ctx->stream));
  if (n > 0) CK(cudaMemcpyAsync(d, host_bits, (size_t)((n + 7) / 8), cudaMemcpyHostToDevice, ctx->stream));
  *out = d;
  return QM_OK;
}

// Host bytes to device memory on the context's stream: page-locked and small
// sources by one copy, large pageable ones staged through pinned buffers by
// host threads (defined with the page ingest).
int upload_host_bytes(qm_ctx *ctx, const void *src, size_t n, void *dst);

int make_col(qm_ctx *ctx, int64_t n, const qm_column &src, DevCol &c) {
  if (!src.name) return set_err(ctx, QM_ERR_INVALID, "column without a name");
  if (!valid_dtype(src.dtype))
    return set_err(ctx, QM_ERR_UNSUPPORTED, "column %s: dtype %d is not numeric", src.name, src.dtype);
  c.name = src.name;
  c.dtype = src.dtype;
  if (n > 0 && !src.data) return set_err(ctx, QM_ERR_INVALID, "column %s: no data", src.name);
  if (src.on_device) {
    c.data = const_cast<void *>(src.data);
    if (src.null_bitmap) {
      // a device bitmap must already be readable as 32-bit words: copy it
      // into an owned, word-padded buffer
      size_t words = (size_t)((n + 31) / 32) + 1;
      uint32_t *d = (uint32_t *)col_alloc(ctx, words * 4, c.nulls_block);
      if (!d) return set_err(ctx, QM_ERR_OOM, "null bitmap alloc (%zu bytes)", words * 4);
      c.nulls = d;
      c.own_nulls = true;
      CK(cudaMemsetAsync(d, 0, words * 4, ctx->stream));
      if (n > 0)
        CK(cudaMemcpyAsync(d, src.null_bitmap, (size_t)((n + 7) / 8), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return QM_OK;
  }
  size_t bytes = (size_t)n * dtype_size(src.dtype);
  void *d = col_alloc(ctx, std::max<size_t>(bytes, 16), c.data_block);
  if (!d) return set_err(ctx, QM_ERR_OOM, "column %s: device memory (%zu bytes)", src.name, bytes);
  c.data = d;
  c.own_data = true;
  if (bytes) {
    int rc = upload_host_bytes(ctx, src.data, bytes, d);
    if (rc) return rc;
  }
  if (src.null_bitmap) {
    c.own_nulls = true;
    int rc = upload_nulls(ctx, src.null_bitmap, n, &c.nulls, c.nulls_block);
    if (rc) return rc;
  }
  return QM_OK;
}

// ------------------------------------------------------------ planning
struct ColView {  // what the planner needs to know of a column
  const DevCol *col;
  int64_t n;
};

struct OutMeta {
  std::string name;
  int dtype;
  int is_key;
  bool nullable;
};

struct Plan {
  qm_pred pred{};
  qm_keyspec key{};
  qm_aggspec agg{};
  qm_outspec outs{};
  std::vector<OutMeta> meta;
  int64_t bytes_per_row = 0;  // algorithmic: widths of referenced columns
  bool ordered = true;
  int key_col_dtype = 0;
  const DevCol *keycols[QM_MAX_KEYS] = {nullptr, nullptr, nullptr, nullptr};
  const DevCol *vcolsrc[QM_MAX_VCOLS] = {};
  // post-aggregate ORDER BY / LIMIT / OFFSET: 0 none, 1 first-seen slice,
  // 2 stable sort (then OFFSET), 3 TopK heap (LIMIT + OFFSET rows, then OFFSET)
  int post = 0;
  int post_col = -1;  // output column sorted by; -1: a name no output has
  int post_desc = 0;
  int post_has_limit = 0;
  int64_t post_limit = 0, post_offset = 0;
};

const i128 BIG = (i128)1 << 100;

i128 clamp_d(double d) {  // integer-valued double -> i128, saturating
  if (d >= 1e30) return BIG;
  if (d <= -1e30) return -BIG;
  return (i128)d;
}

// A JS comparison threshold as seen from an integer cell.  kind: 0 finite
// (floor/ceil exact integers), 1 NaN.  ±Infinity are finite beyond any
// int64 (±2^101).
struct Thr {
  int nan = 0;
  i128 fl = 0, ce = 0;
};

Thr thr_of_number_exact(double t) {  // int32 cell (a JS number) vs number t
  Thr r;
  if (std::isnan(t)) {
    r.nan = 1;
    return r;
  }
  if (std::isinf(t)) {
    r.fl = r.ce = t > 0 ? BIG * 2 : -BIG * 2;
    return r;
  }
  r.fl = clamp_d(std::floor(t));
  r.ce = clamp_d(std::ceil(t));
  return r;
}

Thr thr_of_int(i128 T) {
  Thr r;
  r.fl = r.ce = T;
  return r;
}

// ECMAScript ToInt32 (a number passed as a WASM i32 parameter).
int32_t to_int32(double x) {
  if (!std::isfinite(x)) return 0;
  double t = std::trunc(x);
  double m = std::fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}

// safeBigInt then ToBigInt64 (a bigint passed as a WASM i64 parameter).
int64_t to_wasm_i64(double x) {
  if (!std::isfinite(x)) return 0;
  double t = std::trunc(x);
  if (std::fabs(t) < 9.2e18) return (int64_t)t;
  double m = std::fmod(t, 18446744073709551616.0);
  if (m < 0) m += 18446744073709551616.0;
  uint64_t u = m >= 9223372036854775808.0 ? (uint64_t)(m - 9223372036854775808.0) + 9223372036854775808ULL
                                           : (uint64_t)m;
  return (int64_t)u;
}

// The threshold an integer cell is compared with, after JS coercion.
Thr int_threshold(int dtype, const qm_value &v, bool wasm) {
  if (v.kind == QM_VAL_BIGINT) return thr_of_int((i128)v.big);
  if (wasm) {
    if (dtype == QM_I32) return thr_of_int((i128)to_int32(v.num));
    return thr_of_int((i128)to_wasm_i64(v.num));
  }
  if (dtype == QM_I64) {
    // bigint cell: BigInt(Math.trunc(t)) for finite t, else the number
    if (std::isfinite(v.num)) return thr_of_int(clamp_d(std::trunc(v.num)));
    return thr_of_number_exact(v.num);
  }
  return thr_of_number_exact(v.num);
}

struct IRange {
  int konst = -1;  // -1: a range test; 0 / 1: constant result
  bool negate = false;
  i128 lo = 0, hi = 0;
};

IRange int_range_for(int op, const Thr &t) {
  IRange r;
  if (t.nan) {
    r.konst = op == QM_OP_NEQ ? 1 : 0;
    return r;
  }
  const i128 MIN = -BIG * 4, MAX = BIG * 4;
  switch (op) {
    case QM_OP_EQ: if (t.fl != t.ce) { r.konst = 0; return r; } r.lo = r.hi = t.fl; break;
    case QM_OP_NEQ: if (t.fl != t.ce) { r.konst = 1; return r; } r.lo = r.hi = t.fl; r.negate = true; break;
    case QM_OP_LT: r.lo = MIN; r.hi = t.ce - 1; break;
    case QM_OP_LTE: r.lo = MIN; r.hi = t.fl; break;
    case QM_OP_GT: r.lo = t.fl + 1; r.hi = MAX; break;
    default: r.lo = t.ce; r.hi = MAX; break;  // GTE
  }
  return r;
}

bool range_test0(const IRange &r) {  // does the test pass for the value 0?
  if (r.konst >= 0) return r.konst;
  bool in = r.lo <= 0 && 0 <= r.hi;
  return r.negate ? !in : in;
}

void lower_irange(const IRange &r0, int dtype, qm_term &t) {
  IRange r = r0;
  const i128 dmin = dtype == QM_I32 ? (i128)INT32_MIN : (i128)INT64_MIN;
  const i128 dmax = dtype == QM_I32 ? (i128)INT32_MAX : (i128)INT64_MAX;
  if (r.konst >= 0) {
    t.kind = r.konst ? QT_TRUE : QT_FALSE;
    return;
  }
  i128 lo = std::max(r.lo, dmin), hi = std::min(r.hi, dmax);
  bool empty = lo > hi;
  bool full = !empty && lo == dmin && hi == dmax;
  if (!r.negate) {
    if (empty) { t.kind = QT_FALSE; return; }
    if (full) { t.kind = QT_TRUE; return; }
    t.kind = QT_IRANGE;
  } else {
    if (empty) { t.kind = QT_TRUE; return; }
    if (full) { t.kind = QT_FALSE; return; }
    t.kind = QT_INRANGE;
  }
  t.lo = (int64_t)lo;
  t.hi = (int64_t)hi;
}

// Does the scan-time WASM filter (applyAndFilters, src/operators.ts:469-547)
// take its WASM branch for this filter?
bool wasm_route(int dtype, const qm_filter &f) {
  if (f.op <= QM_OP_GTE) {
    if (f.value.kind != QM_VAL_NUMBER) return false;
    if (dtype == QM_I64 && !std::isfinite(f.value.num)) return false;
    return true;
  }
  if (f.op == QM_OP_BETWEEN || f.op == QM_OP_NOT_BETWEEN) {
    if (f.value.kind != QM_VAL_NUMBER || f.value2.kind != QM_VAL_NUMBER) return false;
    if (dtype == QM_I64 && (!std::isfinite(f.value.num) || !std::isfinite(f.value2.num))) return false;
    return true;
  }
  return false;
}

bool fcmp_host(double v, int op, double t) {
  switch (op) {
    case 0: return v == t; case 1: return v != t; case 2: return v < t;
    case 3: return v <= t; case 4: return v > t; default: return v >= t;
  }
}

int lower_filter(qm_ctx *ctx, const qm_filter &f, const ColView &cv, bool wasm_flag, qm_term &t) {
  const DevCol &c = *cv.col;
  memset(&t, 0, sizeof t);
  t.data = c.data;
  t.nulls = c.nulls;
  t.dtype = c.dtype;
  t.null_pass = 0;
  if (f.op == QM_OP_IS_NULL) { t.kind = QT_FALSE; t.null_pass = 1; return QM_OK; }
  if (f.op == QM_OP_IS_NOT_NULL) { t.kind = QT_TRUE; t.null_pass = 0; return QM_OK; }
  if (f.op < 0 || f.op > QM_OP_NOT_BETWEEN)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "filter op %d on %s is not on the GPU path", f.op, c.name.c_str());
  if (f.value.kind != QM_VAL_NUMBER && f.value.kind != QM_VAL_BIGINT)
    return set_err(ctx, QM_ERR_INVALID, "filter on %s: bad value kind", c.name.c_str());
  const bool wasm = wasm_flag && wasm_route(c.dtype, f);
  const bool range = f.op == QM_OP_BETWEEN || f.op == QM_OP_NOT_BETWEEN;
  if (is_int(c.dtype)) {
    IRange r;
    if (!range) {
      r = int_range_for(f.op, int_threshold(c.dtype, f.value, wasm));
    } else {
      if (f.value2.kind != QM_VAL_NUMBER && f.value2.kind != QM_VAL_BIGINT)
        return set_err(ctx, QM_ERR_INVALID, "filter on %s: bad BETWEEN bound", c.name.c_str());
      Thr a = int_threshold(c.dtype, f.value, wasm), b = int_threshold(c.dtype, f.value2, wasm);
      if (f.op == QM_OP_BETWEEN) {  // v >= a && v <= b (inclusive)
        if (a.nan || b.nan) r.konst = 0;
        else { r.lo = a.ce; r.hi = b.fl; }
      } else {                      // v < a || v > b
        if (a.nan && b.nan) r.konst = 0;
        else if (a.nan) { r.lo = b.fl + 1; r.hi = BIG * 4; }
        else if (b.nan) { r.lo = -BIG * 4; r.hi = a.ce - 1; }
        else { r.lo = a.ce; r.hi = b.fl; r.negate = true; }
      }
    }
    lower_irange(r, c.dtype, t);
    if (wasm) t.null_pass = range_test0(r) ? 1 : 0;  // WASM reads a NULL cell as 0
    return QM_OK;
  }
  // float column (JS number cells)
  if (!range) {
    if (f.value.kind == QM_VAL_BIGINT) {
      t.kind = QT_FBIG;
      t.op = f.op;
      t.lo = f.value.big;
      return QM_OK;
    }
    const double v = f.value.num;
    if (wasm) t.null_pass = fcmp_host(0.0, f.op, v) ? 1 : 0;
    if (f.op == QM_OP_NEQ) {
      t.kind = QT_FCMP;
      t.op = f.op;
      t.f0 = v;
      return QM_OK;
    }
    if (std::isnan(v)) {  // every comparison with NaN is false
      t.kind = QT_FALSE;
      return QM_OK;
    }
    // float ranges are kept inclusive: for a non-NaN cell, v > x is
    // v >= nextafter(x, +inf) and v < x is v <= nextafter(x, -inf)
    t.kind = QT_FRANGE;
    t.f0 = -INFINITY;
    t.f1 = INFINITY;
    t.op = 3;
    switch (f.op) {
      case QM_OP_EQ: t.f0 = t.f1 = v; break;
      case QM_OP_LT:
        if (v == -INFINITY) t.kind = QT_FALSE;
        else t.f1 = std::nextafter(v, -INFINITY);
        break;
      case QM_OP_LTE: t.f1 = v; break;
      case QM_OP_GT:
        if (v == INFINITY) t.kind = QT_FALSE;
        else t.f0 = std::nextafter(v, INFINITY);
        break;
      default: t.f0 = v; break;  // GTE
    }
    return QM_OK;
  }
  if (f.value.kind != QM_VAL_NUMBER || f.value2.kind != QM_VAL_NUMBER)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "BETWEEN with bigint bounds on float column %s", c.name.c_str());
  t.kind = f.op == QM_OP_BETWEEN ? QT_FRANGE : QT_FNBETWEEN;
  t.op = 3;
  t.f0 = f.value.num;
  t.f1 = f.value2.num;
  if (f.op == QM_OP_BETWEEN && (std::isnan(t.f0) || std::isnan(t.f1))) t.kind = QT_FALSE;
  if (wasm) {
    bool p = f.op == QM_OP_BETWEEN ? (0.0 >= t.f0 && 0.0 <= t.f1) : (0.0 < t.f0 || 0.0 > t.f1);
    t.null_pass = p ? 1 : 0;
  }
  return QM_OK;
}

typedef const ColView *(*Resolver)(void *env, const char *name);

struct ColEnv {
  std::vector<ColView> views;
  const ColView *find(const char *name) const {
    for (auto &v : views)
      if (v.col->name == name) return &v;
    return nullptr;
  }
};

int build_pred(qm_ctx *ctx, const qm_query *q, const ColEnv &env, qm_pred &P, int64_t &bytes_per_row,
               std::vector<const DevCol *> &touched) {
  memset(&P, 0, sizeof P);
  const bool wasm = (q->flags & QM_FLAG_WASM_SCAN_SEMANTICS) != 0;
  int nt = 0;
  if (q->n_filters < 0 || q->n_or_groups < 0) return set_err(ctx, QM_ERR_INVALID, "negative filter count");
  auto add = [&](const qm_filter &f) -> int {
    if (nt >= QM_MAX_TERMS) return set_err(ctx, QM_ERR_UNSUPPORTED, "more than %d filter terms", QM_MAX_TERMS);
    if (!f.column) return set_err(ctx, QM_ERR_INVALID, "filter without a column");
    const ColView *cv = env.find(f.column);
    if (!cv) return set_err(ctx, QM_ERR_NOT_FOUND, "unknown filter column %s", f.column);
    int rc = lower_filter(ctx, f, *cv, wasm, P.t[nt]);
    if (rc) return rc;
    if (std::find(touched.begin(), touched.end(), cv->col) == touched.end()) touched.push_back(cv->col);
    nt++;
    return QM_OK;
  };
  for (int i = 0; i < q->n_filters; i++) {
    int rc = add(q->filters[i]);
    if (rc) return rc;
    // AND-ed range tests on one column become one test (one read per row)
    qm_term &nw = P.t[nt - 1];
    for (int j = 0; j < nt - 1; j++) {
      qm_term &o = P.t[j];
      if (o.data != nw.data || o.kind != nw.kind || o.dtype != nw.dtype) continue;
      if (nw.kind == QT_IRANGE) {
        o.lo = std::max(o.lo, nw.lo);
        o.hi = std::min(o.hi, nw.hi);
        if (o.lo > o.hi) o.kind = QT_FALSE;
      } else if (nw.kind == QT_FRANGE) {  // inclusive bounds
        o.f0 = std::max(o.f0, nw.f0);
        o.f1 = std::min(o.f1, nw.f1);
      } else {
        continue;
      }
      o.null_pass = o.null_pass && nw.null_pass;
      nt--;
      break;
    }
  }
  P.n_and = nt;
  int off = 0;
  for (int g = 0; g < q->n_or_groups; g++) {
    int sz = q->or_group_sizes[g];
    if (sz < 0) return set_err(ctx, QM_ERR_INVALID, "negative OR group size");
    for (int i = 0; i < sz; i++) {
      int rc = add(q->or_filters[off + i]);
      if (rc) return rc;
    }
    off += sz;
    P.group_end[g] = nt;
  }
  P.n_groups = q->n_or_groups;
  if (P.n_groups > QM_MAX_TERMS) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many OR groups");
  (void)bytes_per_row;
  return QM_OK;
}

const char *agg_name(int fn) {
  static const char *n[] = {"sum", "avg", "min", "max", "count"};
  return (fn >= 0 && fn <= 4) ? n[fn] : "?";
}

// Builds the key spec (without the mode), the accumulators and the outputs.
int build_agg(qm_ctx *ctx, const qm_query *q, const ColEnv &env, Plan &pl, std::vector<const DevCol *> &touched) {
  qm_keyspec &K = pl.key;
  qm_aggspec &A = pl.agg;
  memset(&K, 0, sizeof K);
  memset(&A, 0, sizeof A);
  pl.meta.clear();
  if (q->n_group_by < 0 || q->n_aggregates < 0) return set_err(ctx, QM_ERR_INVALID, "negative counts");
  if (q->n_group_by > QM_MAX_KEYS)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "GROUP BY over more than %d columns", QM_MAX_KEYS);
  const DevCol *kc[QM_MAX_KEYS] = {nullptr, nullptr, nullptr, nullptr};
  for (int i = 0; i < q->n_group_by; i++) {
    if (!q->group_by[i]) return set_err(ctx, QM_ERR_INVALID, "group column without a name");
    const ColView *cv = env.find(q->group_by[i]);
    if (!cv) return set_err(ctx, QM_ERR_NOT_FOUND, "unknown group column %s", q->group_by[i]);
    kc[i] = cv->col;
    if (std::find(touched.begin(), touched.end(), cv->col) == touched.end()) touched.push_back(cv->col);
  }
  K.n_cols = q->n_group_by;
  for (int i = 0; i < K.n_cols; i++) {
    K.data[i] = kc[i]->data;
    K.nulls[i] = kc[i]->nulls;
    K.dtype[i] = kc[i]->dtype;
    pl.keycols[i] = kc[i];
  }
  K.pack = QP_RAW;  // multi-column packing is chosen with the key mode
  // accumulators
  auto add_acc = [&](int kind, int vcol, int wide) -> int {
    for (int i = 0; i < A.n_accs; i++)
      if (A.acc[i].kind == kind && A.acc[i].vcol == vcol) return i;
    if (A.n_accs >= QM_MAX_ACCS) return -1;
    int width = (kind == QA_ISUM || kind == QA_FSUM) ? 2 : 1;
    if (A.n_words + width > QM_MAX_WORDS) return -1;
    qm_acc &a = A.acc[A.n_accs];
    a.kind = kind;
    a.vcol = vcol;
    a.word = A.n_words;
    a.wide = wide;
    a.narrow = 0;
    a.pad = 0;
    uint64_t init = 0;
    switch (kind) {
      case QA_FIRST: case QA_FZERO: init = ~0ULL; break;
      case QA_IMIN: init = (uint64_t)INT64_MAX; break;
      case QA_IMAX: init = (uint64_t)INT64_MIN; break;
      case QA_FMIN: init = (uint64_t)qm_f2ord_host(INFINITY); break;
      case QA_FMAX: init = (uint64_t)qm_f2ord_host(-INFINITY); break;
      default: init = 0;
    }
    for (int w = 0; w < width; w++) A.init[A.n_words + w] = init;
    A.n_words += width;
    return A.n_accs++;
  };
  A.acc_count = add_acc(QA_COUNT, -1, 0);
  pl.ordered = (q->flags & QM_FLAG_UNORDERED) == 0;
  A.acc_first = pl.ordered && K.n_cols > 0 ? add_acc(QA_FIRST, -1, 0) : -1;
  std::vector<const DevCol *> vcols;
  auto vcol_of = [&](const DevCol *c) -> int {
    for (size_t i = 0; i < vcols.size(); i++)
      if (vcols[i] == c) return (int)i;
    if ((int)vcols.size() >= QM_MAX_VCOLS) return -1;
    vcols.push_back(c);
    pl.vcolsrc[vcols.size() - 1] = c;
    A.vcol[vcols.size() - 1].split = 0.0;
    A.vcol[vcols.size() - 1].data = c->data;
    A.vcol[vcols.size() - 1].nulls = c->nulls;
    A.vcol[vcols.size() - 1].dtype = c->dtype;
    return (int)vcols.size() - 1;
  };
  // outputs: keys, then aggregates in query order
  qm_outspec &O = pl.outs;
  memset(&O, 0, sizeof O);
  for (int i = 0; i < K.n_cols; i++) {
    qm_out &o = O.o[O.n_out++];
    o.kind = QO_KEY;
    o.src = i;
    o.dtype = kc[i]->dtype == QM_F32 ? QM_F64 : kc[i]->dtype;
    o.zero_word = -1;
    pl.meta.push_back({q->group_by[i], o.dtype, 1, kc[i]->nulls != nullptr});
  }
  if (K.n_cols + q->n_aggregates > QM_MAX_OUT) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many output columns");
  for (int i = 0; i < q->n_aggregates; i++) {
    const qm_aggregate &ag = q->aggregates[i];
    if (!ag.column) return set_err(ctx, QM_ERR_INVALID, "aggregate without a column");
    if (ag.fn < QM_AGG_SUM || ag.fn > QM_AGG_COUNT)
      return set_err(ctx, QM_ERR_UNSUPPORTED, "aggregate fn %d is not on the GPU path", ag.fn);
    std::string name = ag.alias ? std::string(ag.alias) : std::string(agg_name(ag.fn)) + "_" + ag.column;
    qm_out &o = O.o[O.n_out++];
    memset(&o, 0, sizeof o);
    o.zero_word = -1;
    o.nn_word = A.acc[A.acc_count].word;
    const bool star = strcmp(ag.column, "*") == 0;
    if (star) {
      if (ag.fn != QM_AGG_COUNT) return set_err(ctx, QM_ERR_INVALID, "%s(*) is not an aggregate", agg_name(ag.fn));
      o.kind = QO_COUNT;
      o.dtype = QM_I64;
      o.word = A.acc[A.acc_count].word;
      pl.meta.push_back({name, o.dtype, 0, false});
      continue;
    }
    const ColView *cv = env.find(ag.column);
    if (!cv) return set_err(ctx, QM_ERR_NOT_FOUND, "unknown aggregate column %s", ag.column);
    const DevCol *c = cv->col;
    if (std::find(touched.begin(), touched.end(), c) == touched.end()) touched.push_back(c);
    int vc = vcol_of(c);
    if (vc < 0) return set_err(ctx, QM_ERR_UNSUPPORTED, "more than %d aggregated columns", QM_MAX_VCOLS);
    int nn_acc = c->nulls ? add_acc(QA_NN, vc, 0) : A.acc_count;
    if (nn_acc < 0) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many accumulators");
    o.nn_word = A.acc[nn_acc].word;
    int acc = -1;
    switch (ag.fn) {
      case QM_AGG_COUNT:
        o.kind = QO_COUNT;
        o.dtype = QM_I64;
        o.word = o.nn_word;
        break;
      case QM_AGG_SUM:
      case QM_AGG_AVG:
        if (is_int(c->dtype)) {
          acc = add_acc(QA_ISUM, vc, c->dtype == QM_I64);
          if (c->dtype == QM_I64) {
            o.kind = ag.fn == QM_AGG_SUM ? QO_SUM_I128 : QO_AVG_BIG;
            o.dtype = ag.fn == QM_AGG_SUM ? QM_I128 : QM_F64;
          } else {
            o.kind = ag.fn == QM_AGG_SUM ? QO_SUM_I2F : QO_AVG_I2F;
            o.dtype = QM_F64;
          }
        } else {
          acc = add_acc(QA_FSUM, vc, 0);
          o.kind = ag.fn == QM_AGG_SUM ? QO_SUM_F : QO_AVG_F;
          o.dtype = QM_F64;
          if (q->flags & QM_FLAG_DETERMINISTIC) {
            // fixed-point sum: its non-finite cells go to a word of their own
            const int nf = add_acc(QA_FNF, vc, 0);
            if (nf < 0) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many accumulators");
            o.fixed = 1;
            o.nf_word = A.acc[nf].word;
          }
        }
        break;
      case QM_AGG_MIN:
      case QM_AGG_MAX:
        if (is_int(c->dtype)) {
          acc = add_acc(ag.fn == QM_AGG_MIN ? QA_IMIN : QA_IMAX, vc, 0);
          o.kind = ag.fn == QM_AGG_MIN ? QO_MIN_I : QO_MAX_I;
          o.dtype = c->dtype;
        } else {
          acc = add_acc(ag.fn == QM_AGG_MIN ? QA_FMIN : QA_FMAX, vc, 0);
          int z = add_acc(QA_FZERO, vc, 0);
          if (z < 0) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many accumulators");
          o.zero_word = A.acc[z].word;
          o.kind = ag.fn == QM_AGG_MIN ? QO_MIN_F : QO_MAX_F;
          o.dtype = QM_F64;
        }
        break;
    }
    if (ag.fn != QM_AGG_COUNT) {
      if (acc < 0) return set_err(ctx, QM_ERR_UNSUPPORTED, "too many accumulators");
      o.word = A.acc[acc].word;
    }
    pl.meta.push_back({name, o.dtype, 0, ag.fn != QM_AGG_COUNT});
  }
  A.n_vcols = (int)vcols.size();
  A.w_count = A.acc[A.acc_count].word;
  A.w_first = A.acc_first >= 0 ? A.acc[A.acc_first].word : -1;
  for (int c = 0; c < A.n_vcols; c++) {
    qm_vcol &vc = A.vcol[c];
    vc.flags = 0;
    vc.w_nn = vc.w_sum = vc.w_min = vc.w_max = vc.w_zero = vc.w_nf = -1;
    vc.fx_exp = 0;
    vc.fx_max = 0.0;
  }
  for (int i = 0; i < A.n_accs; i++) {
    const qm_acc &ac = A.acc[i];
    if (ac.vcol < 0) continue;
    qm_vcol &vc = A.vcol[ac.vcol];
    switch (ac.kind) {
      case QA_NN: vc.flags |= VF_NN; vc.w_nn = ac.word; break;
      case QA_ISUM: vc.flags |= VF_SUM | (ac.wide ? VF_WIDE : 0); vc.w_sum = ac.word; break;
      case QA_FSUM: vc.flags |= VF_SUM; vc.w_sum = ac.word; break;
      case QA_IMIN: case QA_FMIN: vc.flags |= VF_MIN; vc.w_min = ac.word; break;
      case QA_IMAX: case QA_FMAX: vc.flags |= VF_MAX; vc.w_max = ac.word; break;
      case QA_FZERO: vc.flags |= VF_ZERO; vc.w_zero = ac.word; break;
      case QA_FNF: vc.w_nf = ac.word; break;
    }
  }
  return QM_OK;
}

// ------------------------------------------------------------ execution
struct Exec {
  int64_t n_slots = 1;  // QK_DIRECT size / QK_HASH capacity
  int log2cap = 0;
  int64_t total_slots = 1;
  int stride = 1;
  int local_slots = 0;
  int local_hash = 0;
  int dedupe = 1;
  int strategy = 0;
  int priv = 0;  // direct block-local table copied per warp (no atomics)
};

int64_t special_slots(int mode) { return mode == QK_HASH ? 2 : (mode == QK_DIRECT ? 1 : 0); }

int ilog2_ceil(int64_t x) {
  int l = 0;
  while (((int64_t)1 << l) < x) l++;
  return l;
}

constexpr size_t LOCAL_BUDGET = 40 * 1024;  // bytes of the block-local hash table
constexpr size_t LOCAL_WIDE_BUDGET = 80 * 1024;  // ... when the estimated groups overflow it
constexpr int64_t LOCAL_WIDE_MAX_GROUPS = 10000;
// A dense (direct) key range whose table fits this many bytes is aggregated
// entirely in shared memory, even at one block per SM: every row then stays
// on the shared-memory path instead of the L2 atomics of the global table.
constexpr size_t DIRECT_LOCAL_BUDGET = 180 * 1024;
// Bytes of all per-warp copies of a small direct table.
constexpr size_t PRIV_BUDGET = 64 * 1024;
constexpr int64_t PRIV_MIN_ROWS = (int64_t)8 << 20;

void choose_layout(const Plan &pl, int64_t est_groups, Exec &ex, const qm_tuning &tu) {
  const int words = pl.agg.n_words;
  ex.stride = 1 + words;
  ex.total_slots = ex.n_slots + special_slots(pl.key.mode);
  const int64_t per_slot = (int64_t)words * 8;
  ex.priv = 0;
  if (pl.key.mode == QK_NONE) {
    ex.local_slots = 1;
    ex.local_hash = 0;
    ex.dedupe = 1;
    ex.priv = 1;
    ex.strategy = 0;
    return;
  }
  if (pl.key.mode == QK_DIRECT && tu.local_slots >= 0 && (ex.n_slots + 1) * per_slot <= (int64_t)DIRECT_LOCAL_BUDGET) {
    ex.local_slots = (int)(ex.n_slots + 1);
    ex.local_hash = 0;
    // warp deduplication is off by default for dense keys: the scan's own
    // equal-slot merge costs fewer instructions (measured 2.5x faster at 11
    // groups, 1.5x at 16)
    ex.dedupe = tu.dedupe >= 0 ? tu.dedupe : 0;
    // deduplicated rows have distinct slots within a warp, so a small table
    // copied per warp is then updated without atomics
    ex.priv = ex.dedupe && (ex.n_slots + 1) * per_slot * (QM_SCAN_THREADS / 32) <= (int64_t)PRIV_BUDGET;
    ex.strategy = 0;
    return;
  }
  if (tu.local_slots > 0 || (tu.local_slots == 0 && est_groups <= ((int64_t)1 << 20))) {
    int L = 1;
    while ((int64_t)(L * 2) * (per_slot + 8) <= (int64_t)LOCAL_BUDGET) L *= 2;
    // More groups than that table admits (half its slots): a wider table,
    // still two blocks per SM, keeps them in shared memory (256-1,000
    // int64 groups at 75 % selectivity: 3.9 -> 1.9 ms over 15 queries).
    if (tu.local_slots == 0 && est_groups > L / 2 && est_groups <= LOCAL_WIDE_MAX_GROUPS)
      while ((int64_t)(L * 2) * (per_slot + 8) <= (int64_t)LOCAL_WIDE_BUDGET) L *= 2;
    if (tu.local_slots > 0) {
      L = tu.local_slots;
      while (L > 1 && (int64_t)L * (per_slot + 8) > (int64_t)200 * 1024) L /= 2;  // fit shared memory
    }
    ex.local_slots = L;
    ex.local_hash = 1;
    ex.dedupe = tu.dedupe >= 0 ? tu.dedupe : 0;
    ex.strategy = 1;
    return;
  }
  ex.local_slots = 0;
  ex.local_hash = 0;
  ex.dedupe = tu.dedupe >= 0 ? tu.dedupe : 0;
  ex.strategy = 2;
}

std::mutex g_cfg_mu;
// Occupancy answers are fixed per (device, kernel, shared memory) and the
// runtime queries cost tens of microseconds under g_cfg_mu, which every
// planning thread takes: they are cached.  Kernel ids: -1 / -2 the generic
// scan (direct / staged), >= 0 a batched class.
std::map<std::tuple<int, int, size_t>, int> g_occ;
// The largest dynamic shared-memory limit set on each batched class kernel:
// the limit is only ever raised, so a lane never lowers it under another
// lane's larger launch.
std::map<std::pair<int, int>, size_t> g_class_attr;

// cap: blocks per SM for this launch unless the context's tuning sets them.
int scan_blocks(qm_ctx *ctx, size_t smem, int64_t n, bool staged, int cap = 0) {
  int bps = 1;
  {
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    const auto key = std::make_tuple(ctx->device, staged ? -2 : -1, smem);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) {
      bps = it->second;
    } else if (qm_scan_configure(smem, staged, &bps) != cudaSuccess) {
      cudaGetLastError();
      bps = 1;
    } else {
      g_occ[key] = bps;
    }
  }
  if (bps < 1) bps = 1;
  if (ctx->tuning.blocks_per_sm > 0) {
    if (ctx->tuning.blocks_per_sm < bps) bps = ctx->tuning.blocks_per_sm;
  } else if (cap > 0 && cap < bps) {
    bps = cap;
  }
  int64_t tiles = (n + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  int64_t warps = QM_SCAN_THREADS / 32;
  int64_t need = (tiles + warps - 1) / warps;
  int64_t blocks = std::min<int64_t>((int64_t)ctx->sm_count * bps, std::max<int64_t>(need, 1));
  return (int)blocks;
}

// Filter columns to stream through shared memory: every column a term reads,
// at most QM_MAX_STAGED, each 16-byte aligned (bulk copies need it).
bool setup_staging(qm_pred &P, qm_staging &S, int depth) {
  memset(&S, 0, sizeof S);
  const int nt = P.n_groups > 0 ? P.group_end[P.n_groups - 1] : P.n_and;
  int off = 0;
  for (int i = 0; i < nt; i++) {
    qm_term &t = P.t[i];
    t.sidx = -1;
    if (t.kind <= QT_FALSE) continue;
    int c = 0;
    while (c < S.n && S.data[c] != t.data) c++;
    if (c == S.n) {
      if (S.n == QM_MAX_STAGED || ((uintptr_t)t.data & 15)) {
        S.n = 0;
        return false;
      }
      S.data[c] = t.data;
      S.elem[c] = (int)dtype_size(t.dtype);
      S.off[c] = off;
      off += QM_TILE_ROWS * S.elem[c];
      S.n++;
    }
    t.sidx = c;
  }
  if (S.n == 0) return false;
  S.tile_bytes = off;
  S.depth = depth;
  return true;
}

constexpr size_t SMEM_LIMIT = 227 * 1024;

double hll_estimate(const uint32_t *regs) {
  const int m = 1 << QM_HLL_P;
  double sum = 0;
  int zeros = 0;
  for (int i = 0; i < m; i++) {
    sum += std::ldexp(1.0, -(int)regs[i]);
    zeros += regs[i] == 0;
  }
  double alpha = 0.7213 / (1.0 + 1.079 / m);
  double E = alpha * m * (double)m / sum;
  if (E <= 2.5 * m && zeros > 0) E = m * std::log((double)m / zeros);
  return E;
}

// Distinct-key estimate of `n` rows under key spec K (HyperLogLog).
int estimate_groups(qm_ctx *ctx, const qm_keyspec &K, int64_t n, double *out) {
  int rc = ensure(ctx, ctx->hll, sizeof(uint32_t) << QM_HLL_P);
  if (rc) return rc;
  rc = ensure_host(ctx, ctx->hout, sizeof(uint32_t) << QM_HLL_P);
  if (rc) return rc;
  CK(qm_launch_hll(K, n, (uint32_t *)ctx->hll.p, ctx->sm_count, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hout.p, ctx->hll.p, sizeof(uint32_t) << QM_HLL_P, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *out = hll_estimate((const uint32_t *)ctx->hout.p);
  return QM_OK;
}

// Upper bound on the rows a filtered query selects, from a strided sample
// of the predicate (6 standard deviations above the sampled fraction).
constexpr int SEL_SAMPLES = 1 << 16;

bool has_filter(const qm_pred &P) {
  const int nt = P.n_groups > 0 ? P.group_end[P.n_groups - 1] : P.n_and;
  for (int i = 0; i < nt; i++)
    if (P.t[i].kind != QT_TRUE) return true;
  return false;
}

int selected_rows_bound(qm_ctx *ctx, const qm_pred &P, int64_t n, int64_t *out) {
  int rc = ensure(ctx, ctx->counter, 64);
  if (rc) return rc;
  rc = ensure_host(ctx, ctx->hstatus, 64);
  if (rc) return rc;
  CK(qm_launch_sample_pred(P, n, SEL_SAMPLES, (unsigned long long *)ctx->counter.p, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->counter.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double p = (double)*(const uint64_t *)ctx->hstatus.p / SEL_SAMPLES;
  const double up = std::min(1.0, p + 6.0 * std::sqrt(p * (1.0 - p) / SEL_SAMPLES) + 8.0 / SEL_SAMPLES);
  *out = std::min<int64_t>(n, (int64_t)(up * (double)n) + 4096);
  return QM_OK;
}

// selected_rows_bound, remembered per table and predicate.
int table_sel_bound(qm_ctx *ctx, qm_table *t, const qm_pred &P, int64_t *out) {
  uint64_t h = 0x9e3779b97f4a7c15ULL ^ (uint64_t)t->n_rows;
  const unsigned char *b = reinterpret_cast<const unsigned char *>(&P);
  for (size_t i = 0; i < sizeof P; i++) h = (h ^ b[i]) * 0x100000001b3ULL;
  auto it = t->sel_bounds.find(h);
  if (it != t->sel_bounds.end()) {
    *out = it->second;
    return QM_OK;
  }
  int rc = selected_rows_bound(ctx, P, t->n_rows, out);
  if (rc) return rc;
  if (t->sel_bounds.size() > 4096) t->sel_bounds.clear();
  t->sel_bounds[h] = *out;
  return QM_OK;
}

int column_maxabs(qm_ctx *ctx, DevCol &c, int64_t n) {
  if (c.has_maxabs) return QM_OK;
  int rc = ensure(ctx, ctx->counter, 64);
  if (rc) return rc;
  rc = ensure_host(ctx, ctx->hstatus, 64);
  if (rc) return rc;
  CK(qm_launch_maxabs(c.data, c.dtype, c.nulls, n, (unsigned long long *)ctx->counter.p, ctx->sm_count, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->counter.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  uint64_t b = *(uint64_t *)ctx->hstatus.p;
  memcpy(&c.maxabs, &b, 8);
  c.has_maxabs = true;
  return QM_OK;
}

// Split constants of the float SUM columns of a table query (see qm_vcol),
// or, for a deterministic query, the unit of their fixed-point sums: with
// every finite |x| < 2^e and fewer than 2^R rows, cells become integers
// below 2^F (F = 125 - R) in units of 2^(e - F), so a group's sum stays
// below 2^125 and each cell is off by at most half a unit, 2^(e - F - 1).
int plan_split_sums(qm_ctx *ctx, Plan &pl, int64_t n_rows, bool deterministic) {
  int bits = 1;
  while (bits < 62 && ((int64_t)1 << bits) <= n_rows) bits++;
  const int k = bits + 1;  // a group has fewer than 2^(k-1) rows
  for (int c = 0; c < pl.agg.n_vcols; c++) {
    qm_vcol &vc = pl.agg.vcol[c];
    vc.split = 0.0;
    if (!(vc.flags & VF_SUM) || is_int(vc.dtype)) continue;
    if (!pl.vcolsrc[c]) {
      if (deterministic) return set_err(ctx, QM_ERR_UNSUPPORTED, "deterministic float SUM needs a registered table");
      continue;
    }
    DevCol &col = *const_cast<DevCol *>(pl.vcolsrc[c]);
    int rc = column_maxabs(ctx, col, n_rows);
    if (rc) return rc;
    int e = 0;  // every finite |x| < 2^e
    if (col.maxabs > 0) e = std::ilogb(col.maxabs) + 1;
    if (deterministic) {
      const int F = 125 - bits;
      vc.flags |= VF_FIXED;
      vc.fx_exp = e - F;
      vc.fx_max = std::ldexp(1.0, e);
      for (int o = 0; o < pl.outs.n_out; o++)
        if ((pl.outs.o[o].kind == QO_SUM_F || pl.outs.o[o].kind == QO_AVG_F) && pl.outs.o[o].word == vc.w_sum)
          pl.outs.o[o].fx_exp = vc.fx_exp;
      continue;
    }
    if (e + k > 1000 || e + k < -960) continue;  // keep TwoSum at the ends of the range
    vc.split = 1.5 * std::ldexp(1.0, e + k);
  }
  return QM_OK;
}

int column_minmax(qm_ctx *ctx, DevCol &c, int64_t n) {
  if (c.has_minmax) return QM_OK;
  int rc = ensure(ctx, ctx->counter, 64);
  if (rc) return rc;
  rc = ensure_host(ctx, ctx->hstatus, 64);
  if (rc) return rc;
  CK(qm_launch_minmax(c.data, c.dtype, c.nulls, n, (long long *)ctx->counter.p, ctx->sm_count, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->counter.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  c.mn = ((long long *)ctx->hstatus.p)[0];
  c.mx = ((long long *)ctx->hstatus.p)[1];
  c.has_minmax = true;
  return QM_OK;
}

// Multi-column keys: integer columns as mixed-radix digits of one 64-bit
// word (NULL is digit 0 of a nullable column) when the column ranges are
// known and the product fits; two non-null int32 columns concatenate
// otherwise.  Returns the number of distinct key words (0 = unbounded).
int plan_key_packing(qm_ctx *ctx, Plan &pl, int64_t n_rows, bool have_stats, uint64_t *space) {
  qm_keyspec &K = pl.key;
  *space = 0;
  if (K.n_cols <= 1) {
    K.pack = QP_RAW;
    return QM_OK;
  }
  bool all_int = true;
  for (int i = 0; i < K.n_cols; i++) all_int = all_int && is_int(K.dtype[i]);
  if (all_int && have_stats) {
    unsigned __int128 prod = 1;
    bool fits = true;
    for (int i = 0; i < K.n_cols && fits; i++) {
      DevCol &c = *const_cast<DevCol *>(pl.keycols[i]);
      int rc = column_minmax(ctx, c, n_rows);
      if (rc) return rc;
      const int nullable = c.nulls ? 1 : 0;
      uint64_t radix;
      if (c.mx >= c.mn) {
        unsigned __int128 r = (unsigned __int128)((__int128)c.mx - (__int128)c.mn) + 1 + nullable;
        if (r > ((unsigned __int128)1 << 62)) fits = false;
        radix = (uint64_t)r;
        K.kbase[i] = c.mn;
      } else {  // no non-null value
        radix = 1 + nullable;
        K.kbase[i] = 0;
      }
      K.knullable[i] = nullable;
      K.kradix[i] = radix;
      prod *= radix;
      if (prod > ((unsigned __int128)1 << 62)) fits = false;
    }
    if (fits) {
      uint64_t m = 1;
      for (int i = K.n_cols - 1; i >= 0; i--) {
        K.kmul[i] = m;
        m *= K.kradix[i];
      }
      K.pack = QP_DIGITS;
      *space = (uint64_t)prod;
      return QM_OK;
    }
  }
  if (K.n_cols == 2 && K.dtype[0] == QM_I32 && K.dtype[1] == QM_I32 && !K.nulls[0] && !K.nulls[1]) {
    K.pack = QP_CONCAT;
    return QM_OK;
  }
  return set_err(ctx, QM_ERR_UNSUPPORTED,
                 "GROUP BY over %d columns needs integer columns whose value ranges pack into 62 bits%s",
                 K.n_cols, have_stats ? "" : " (streamed batches: two non-null int32 columns)");
}

}  // namespace

// ------------------------------------------------------------ results
struct qm_result {
  int64_t n_rows = 0;
  struct Col {
    std::string name;
    int dtype;
    int is_key;
    const uint8_t *data = nullptr;   // inside `buf`
    size_t bytes = 0;
    const uint8_t *nulls = nullptr;  // inside `buf`, QMCB bit order
    bool has_nulls = false;
  };
  std::vector<Col> cols;
  qm_stats stats{};
  std::vector<uint8_t> qmcb;
  bool qmcb_built = false;
  std::shared_ptr<PinnedPool> pool;  // returns `buf` on destruction
  HostBuf buf;
  std::shared_ptr<void> shared;      // a batch's packed buffer, shared by its results
  ~qm_result() {
    if (pool) pool->release(buf);
  }
};

namespace {

// Group table state of one aggregation (one-shot query or a stream of pushes).
struct GroupTable {
  Plan pl;
  Exec ex;
  DevBuf own;            // streaming aggregations own their table
  uint64_t *table = nullptr;
  int64_t rows_done = 0;  // global row index of the next pushed row
  int64_t groups_upper = 0;
  int retries = 0;
  unsigned long long selected = 0;
  bool scan_pending = false;  // evs0/evs1 bracket a scan not yet timed
  double scan_ms = 0;         // accumulated scan-kernel time
  int64_t sel_bound = -1;     // planner's sampled bound on selected rows, if taken
  const uint32_t *zones = nullptr;  // kept zones (device), or null: scan every tile
  int64_t n_zone_tiles = 0;
  bool small_rank = false;  // ranked in one block (ctx->perm, the count in franks[0])
};

int read_status(qm_ctx *ctx, qm_status *out) {
  int rc = ensure_host(ctx, ctx->hstatus, sizeof(qm_status));
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->status.p, sizeof(qm_status), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  memcpy(out, ctx->hstatus.p, sizeof(qm_status));
  return QM_OK;
}

// After a synchronize: fold the bracketed scan time into the table's total.
void take_scan_time(qm_ctx *ctx, GroupTable &gt, bool keep) {
  if (!gt.scan_pending) return;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, ctx->evs0, ctx->evs1) != cudaSuccess) {
    cudaGetLastError();
    ms = 0;
  }
  gt.scan_pending = false;
  if (keep) gt.scan_ms += ms;
}

int init_table(qm_ctx *ctx, GroupTable &gt) {
  CK(qm_launch_init_table(gt.table, gt.ex.total_slots, gt.ex.stride, gt.pl.key.mode == QK_HASH, gt.pl.agg,
                          ctx->sm_count, ctx->stream));
  ctx->launches++;
  return QM_OK;
}

void fill_args(const GroupTable &gt, qm_scan_args &a, qm_status *st) {
  memset(&a, 0, sizeof a);
  a.pred = gt.pl.pred;
  a.key = gt.pl.key;
  a.agg = gt.pl.agg;
  a.table = gt.table;
  a.n_slots = gt.ex.n_slots;
  a.stride = gt.ex.stride;
  a.log2cap = gt.ex.log2cap;
  a.local_slots = gt.ex.local_slots;
  a.local_hash = gt.ex.local_hash;
  a.dedupe = gt.ex.dedupe;
  a.priv = gt.ex.priv;
  a.zones = gt.zones;
  a.n_zone_tiles = gt.n_zone_tiles;
  a.max_probe = 1 << 12;
  a.status = st;
  a.vec_ok = 1;
  const int nt = gt.pl.pred.n_groups > 0 ? gt.pl.pred.group_end[gt.pl.pred.n_groups - 1] : gt.pl.pred.n_and;
  for (int i = 0; i < nt; i++)
    if (((uintptr_t)gt.pl.pred.t[i].data & 15) != 0) a.vec_ok = 0;
}

// Finalize the group table into a qm_result (compaction, first-seen order,
// per-group finalize on the device, one copy back).
bool ranked_finish(const GroupTable &gt) {
  return gt.pl.key.mode != QK_NONE && gt.pl.agg.acc_first >= 0;
}

int64_t rank_words(const GroupTable &gt) { return std::max<int64_t>(gt.rows_done, 1) / 32 + 1; }

// First-seen order: a bit per first row, prefix popcounts give the ranks.
// Queues the ranking and a copy of the group count to ctx->hstatus + 32
// (read after the caller's next synchronize).
int launch_rank(qm_ctx *ctx, GroupTable &gt) {
  const Plan &pl = gt.pl;
  const Exec &ex = gt.ex;
  const int64_t bm_words = rank_words(gt);
  int rc;
  gt.small_rank = ex.total_slots <= QM_SMALL_RANK_SLOTS;
  if (gt.small_rank) {
    // a small table is sorted by first row in one block
    if ((rc = ensure(ctx, ctx->perm, sizeof(uint32_t) * QM_SMALL_RANK_SLOTS)) ||
        (rc = ensure(ctx, ctx->franks, 16)) || (rc = ensure_host(ctx, ctx->hstatus, 64)))
      return rc;
    CK(qm_launch_rank_small(gt.table, ex.total_slots, ex.stride, pl.agg.acc[pl.agg.acc_count].word,
                            pl.agg.acc[pl.agg.acc_first].word, (uint32_t *)ctx->perm.p, (uint64_t *)ctx->franks.p,
                            ctx->stream));
    ctx->launches += 1;
    CK(cudaMemcpyAsync((char *)ctx->hstatus.p + 32, ctx->franks.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    return QM_OK;
  }
  size_t tb = 0;
  CK(qm_rank_temp_bytes(bm_words, &tb));
  if ((rc = ensure(ctx, ctx->fbits, (bm_words + 1) * 4)) || (rc = ensure(ctx, ctx->fcounts, (bm_words + 1) * 4)) ||
      (rc = ensure(ctx, ctx->franks, (bm_words + 1) * 8)) || (rc = ensure(ctx, ctx->sort_temp, tb + 16)) ||
      (rc = ensure_host(ctx, ctx->hstatus, 64)))
    return rc;
  CK(qm_launch_rank_first(gt.table, ex.total_slots, ex.stride, pl.agg.acc[pl.agg.acc_count].word,
                          pl.agg.acc[pl.agg.acc_first].word, (uint32_t *)ctx->fbits.p, bm_words,
                          (uint32_t *)ctx->fcounts.p, (uint64_t *)ctx->franks.p, ctx->sort_temp.p, ctx->sort_temp.bytes,
                          ctx->sm_count, ctx->stream));
  ctx->launches += 3;
  CK(cudaMemcpyAsync((char *)ctx->hstatus.p + 32, (uint64_t *)ctx->franks.p + bm_words, 8, cudaMemcpyDeviceToHost,
                     ctx->stream));
  return QM_OK;
}

// Column offsets of a result buffer of G rows (values, then a word bitmap
// of NULLs for a nullable column, each 16-byte aligned); returns its bytes.
size_t result_layout(const Plan &pl, qm_outspec &O, int64_t G) {
  size_t off = 0;
  const size_t null_words_bytes = (size_t)((G + 31) / 32) * 4;
  for (int k = 0; k < O.n_out; k++) {
    O.o[k].offset = (int64_t)off;
    off += ((size_t)G * dtype_size(O.o[k].dtype) + 15) & ~(size_t)15;
    if (pl.meta[k].nullable) {
      O.o[k].null_offset = (int64_t)off;
      off += (null_words_bytes + 15) & ~(size_t)15;
    } else {
      O.o[k].null_offset = -1;
    }
  }
  return off;
}

// ORDER BY / LIMIT / OFFSET over the G emitted rows in ctx->out (layout O):
// the selected rows in output order into ctx->out2 (layout O2, *G2 rows).
int post_aggregate(qm_ctx *ctx, const Plan &pl, const qm_outspec &O, int64_t G, qm_outspec &O2, int64_t *G2,
                   size_t *bytes2) {
  const int64_t off0 = std::min(pl.post_offset, G);
  const uint32_t *idx = nullptr;
  int64_t first = 0, n = 0;
  int rc;
  if (pl.post == 1) {  // LimitOperator: first-seen rows [OFFSET, OFFSET + LIMIT)
    first = off0;
    n = pl.post_has_limit ? std::min<int64_t>(G - off0, pl.post_limit) : G - off0;
  } else if (G > 0) {
    const bool wide = pl.post_col >= 0 && O.o[pl.post_col].dtype == QM_I128;
    if ((rc = ensure(ctx, ctx->post_last, G * 4)) || (rc = ensure(ctx, ctx->post_hi, G * 8)) ||
        (rc = ensure(ctx, ctx->post_lo, G * 8)) || (rc = ensure(ctx, ctx->post_idx, G * 4)))
      return rc;
    if (pl.post_col >= 0) {
      const qm_out &c = O.o[pl.post_col];
      CK(qm_launch_sort_keys((const unsigned char *)ctx->out.p + c.offset,
                             c.null_offset >= 0 ? (const uint32_t *)((const unsigned char *)ctx->out.p + c.null_offset)
                                                : nullptr,
                             c.dtype, pl.post_desc, G, (uint32_t *)ctx->post_last.p, (uint64_t *)ctx->post_hi.p,
                             (uint64_t *)ctx->post_lo.p, (uint32_t *)ctx->post_idx.p, ctx->sm_count, ctx->stream));
    } else {  // no output of that name: every row's value is undefined (compares equal, sorts last)
      CK(cudaMemsetAsync(ctx->post_last.p, 1, G * 4, ctx->stream));
      CK(cudaMemsetAsync(ctx->post_hi.p, 0, G * 8, ctx->stream));
      CK(cudaMemsetAsync(ctx->post_lo.p, 0, G * 8, ctx->stream));
    }
    ctx->launches++;
    if (pl.post == 2) {  // InMemorySortOperator: stable sort, then OFFSET
      if (pl.post_col >= 0) {
        size_t tb = 0;
        CK(qm_stable_sort_rows(nullptr, nullptr, nullptr, wide, G, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                               nullptr, &tb, ctx->sm_count, ctx->stream));
        if ((rc = ensure(ctx, ctx->post_idx2, G * 4)) || (rc = ensure(ctx, ctx->post_k1, G * 8)) ||
            (rc = ensure(ctx, ctx->post_k2, G * 8)) || (rc = ensure(ctx, ctx->post_l1, G * 4)) ||
            (rc = ensure(ctx, ctx->post_l2, G * 4)) || (rc = ensure(ctx, ctx->post_temp, tb + 16)))
          return rc;
        size_t tbytes = ctx->post_temp.bytes;
        CK(qm_stable_sort_rows((const uint32_t *)ctx->post_last.p, (const uint64_t *)ctx->post_hi.p,
                               (const uint64_t *)ctx->post_lo.p, wide, G, (uint32_t *)ctx->post_idx.p,
                               (uint32_t *)ctx->post_idx2.p, (uint64_t *)ctx->post_k1.p, (uint64_t *)ctx->post_k2.p,
                               (uint32_t *)ctx->post_l1.p, (uint32_t *)ctx->post_l2.p, ctx->post_temp.p, &tbytes,
                               ctx->sm_count, ctx->stream));
        ctx->launches += wide ? 7 : 5;
        idx = (const uint32_t *)ctx->post_idx.p;
      }
      first = off0;
      n = G - off0;
    } else {  // TopKOperator: heap of LIMIT + OFFSET rows, then OFFSET
      const int64_t k = pl.post_limit + pl.post_offset;
      const int64_t held = std::min(k, G);
      if ((rc = ensure(ctx, ctx->post_idx2, std::max<int64_t>(held, 1) * 4))) return rc;
      if (G > 0xffffffffLL) return set_err(ctx, QM_ERR_UNSUPPORTED, "ORDER BY over more than 2^32 groups");
      CK(qm_launch_topk((const uint32_t *)ctx->post_last.p, (const uint64_t *)ctx->post_hi.p,
                        (const uint64_t *)ctx->post_lo.p, G, k, (uint32_t *)ctx->post_idx.p,
                        (uint32_t *)ctx->post_idx2.p, ctx->stream));
      ctx->launches++;
      idx = (const uint32_t *)ctx->post_idx2.p;
      first = std::min(pl.post_offset, held);
      n = held - first;
    }
  }
  if (n < 0) n = 0;
  O2 = O;
  *bytes2 = result_layout(pl, O2, n);
  if ((rc = ensure(ctx, ctx->out2, *bytes2 + 16))) return rc;
  CK(cudaMemsetAsync(ctx->out2.p, 0, *bytes2 + 16, ctx->stream));
  CK(qm_launch_gather_rows((const unsigned char *)ctx->out.p, O, O2, idx, first, n, (unsigned char *)ctx->out2.p,
                           ctx->sm_count, ctx->stream));
  if (n > 0) ctx->launches++;
  *G2 = n;
  return QM_OK;
}

// groups_known >= 0: launch_rank already ran and its count was read.
// Results of at most this many bytes laid out for every slot of the table
// are emitted and copied before the status is read (one synchronise per
// query instead of two; finish_table's `spec`).
constexpr size_t SPEC_RESULT_BYTES = (size_t)8 << 20;

// spec (speculative, ranked queries without post-aggregate clauses): the
// result is laid out for every slot of the table, emitted and copied before
// the status has been read; the status (enqueued by the caller into
// ctx->hstatus) and the group count come with the same synchronise.  On a
// device error *out stays null and *spec holds the status: the caller
// regrows and runs again.
// rows_resident: the plan's key columns hold every row the first-row bitmap
// indexes (a query over a resident table), so a large direct-indexed result
// can be emitted in output order by walking that bitmap.  (Not for hash
// tables: the walk's probes and its pass over every row's bitmap word
// measured slower there, 0.73 -> 0.87 ms of finalize at 971K groups; their
// large results take the two ordered steps of qm_launch_emit_perm.)
constexpr int64_t WALK_MIN_SLOTS = (int64_t)1 << 20;
constexpr int64_t EMIT_CHUNK_MIN_ROWS = (int64_t)1 << 22;
// Results of at least this many rows (hashed, or direct ones not walked) are
// emitted in two ordered steps rather than cell by cell at their ranks.
constexpr int64_t PERM_MIN_ROWS = (int64_t)1 << 18;
constexpr int EMIT_CHUNKS = QM_EMIT_CHUNKS;
int finish_table(qm_ctx *ctx, GroupTable &gt, qm_result **out, float scan_ms_so_far, int64_t groups_known = -1,
                 qm_status *spec = nullptr, bool rows_resident = false) {
  const Plan &pl = gt.pl;
  const Exec &ex = gt.ex;
  int64_t G = 0;
  const uint32_t *slots = nullptr;
  const int first_word_o = pl.agg.acc_first >= 0 ? pl.agg.acc[pl.agg.acc_first].word : -1;
  const bool ranked = ranked_finish(gt);
  if (pl.key.mode == QK_NONE) {
    G = 1;  // ungrouped: exactly one row (src/partial-agg.ts:313-320)
  } else if (ranked) {
    if (spec) {
      G = ex.total_slots;  // the layout's rows; the group count comes with the status
    } else if (groups_known >= 0) {
      G = groups_known;
    } else {
      int rc = launch_rank(ctx, gt);
      if (rc) return rc;
      CK(cudaStreamSynchronize(ctx->stream));
      G = (int64_t)*(uint64_t *)((char *)ctx->hstatus.p + 32);
    }
  } else {
    int rc;
    if ((rc = ensure(ctx, ctx->keys, ex.total_slots * 8)) || (rc = ensure(ctx, ctx->slots, ex.total_slots * 4)) ||
        (rc = ensure(ctx, ctx->counter, 64)) || (rc = ensure_host(ctx, ctx->hstatus, 64)))
      return rc;
    CK(cudaMemsetAsync(ctx->counter.p, 0, 8, ctx->stream));
    const int first_word = pl.agg.acc_first >= 0 ? pl.agg.acc[pl.agg.acc_first].word : -1;
    CK(qm_launch_compact(gt.table, ex.total_slots, ex.stride, pl.agg.acc[pl.agg.acc_count].word, first_word,
                         (uint64_t *)ctx->keys.p, (uint32_t *)ctx->slots.p, (unsigned long long *)ctx->counter.p,
                         ctx->sm_count, ctx->stream));
    ctx->launches++;
    CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->counter.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    G = (int64_t)*(unsigned long long *)ctx->hstatus.p;
    slots = (const uint32_t *)ctx->slots.p;
    if (G > 1 && first_word >= 0) {
      if ((rc = ensure(ctx, ctx->keys2, G * 8)) || (rc = ensure(ctx, ctx->slots2, G * 4))) return rc;
      int end_bit = 1;
      while (end_bit < 64 && ((uint64_t)1 << end_bit) <= (uint64_t)std::max<int64_t>(gt.rows_done, 1)) end_bit++;
      size_t tb = 0;
      CK(qm_sort_pairs(nullptr, &tb, (uint64_t *)ctx->keys.p, (uint64_t *)ctx->keys2.p, (uint32_t *)ctx->slots.p,
                       (uint32_t *)ctx->slots2.p, G, end_bit, ctx->stream));
      if ((rc = ensure(ctx, ctx->sort_temp, tb))) return rc;
      tb = ctx->sort_temp.bytes;
      CK(qm_sort_pairs(ctx->sort_temp.p, &tb, (uint64_t *)ctx->keys.p, (uint64_t *)ctx->keys2.p,
                       (uint32_t *)ctx->slots.p, (uint32_t *)ctx->slots2.p, G, end_bit, ctx->stream));
      slots = (const uint32_t *)ctx->slots2.p;
    }
  }
  // output buffer layout
  qm_outspec O = pl.outs;
  size_t off = 0;
  const size_t null_words_bytes = (size_t)((G + 31) / 32) * 4;
  for (int k = 0; k < O.n_out; k++) {
    O.o[k].offset = (int64_t)off;
    off += ((size_t)G * dtype_size(O.o[k].dtype) + 15) & ~(size_t)15;
    if (pl.meta[k].nullable) {
      O.o[k].null_offset = (int64_t)off;
      off += (null_words_bytes + 15) & ~(size_t)15;
    } else {
      O.o[k].null_offset = -1;
    }
  }
  int rc;
  if ((rc = ensure(ctx, ctx->out, off + 16))) return rc;
  HostBuf hbuf;
  if (!ctx->pool->acquire(off + 16, hbuf)) return set_err(ctx, QM_ERR_OOM, "pinned result buffer (%zu bytes)", off + 16);
  qm_result *R = new qm_result();
  R->pool = ctx->pool;
  R->buf = hbuf;
  // NULL flags are set bit by bit: clear the bitmaps (every data cell of the
  // G rows is written by the emit)
  for (int k = 0; k < O.n_out; k++)
    if (O.o[k].null_offset >= 0)
      CK(cudaMemsetAsync((char *)ctx->out.p + O.o[k].null_offset, 0, null_words_bytes, ctx->stream));
  const bool walk = ranked && !gt.small_rank && rows_resident && pl.key.mode == QK_DIRECT && ex.n_slots >= WALK_MIN_SLOTS;
  // a large result laid out before its group count is known is emitted in
  // chunks of rows, each chunk's copy to host memory running while the next
  // chunk is emitted
  const bool chunked = walk && spec && !pl.post && G >= EMIT_CHUNK_MIN_ROWS;
  if (chunked) {
    if ((rc = ensure(ctx, ctx->wbounds, sizeof(int64_t) * (EMIT_CHUNKS + 1)))) {
      delete R;
      return rc;
    }
    if (!ctx->copy) {
      CK(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
      for (cudaEvent_t &e : ctx->copy_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    qm_scan_args a;
    fill_args(gt, a, (qm_status *)ctx->status.p);
    const int64_t per = ((G + EMIT_CHUNKS - 1) / EMIT_CHUNKS + 31) & ~(int64_t)31;  // whole NULL-bitmap words
    const int64_t words = rank_words(gt);
    const uint64_t *franks = (const uint64_t *)ctx->franks.p;
    CK(qm_launch_walk_bounds(franks, words, per, EMIT_CHUNKS, (int64_t *)ctx->wbounds.p, ctx->stream));
    for (int c = 0; c < EMIT_CHUNKS; c++) {
      const int64_t r0 = std::min<int64_t>(G, c * per), r1 = std::min<int64_t>(G, r0 + per);
      CK(qm_launch_emit_walk(a, (const uint32_t *)ctx->fbits.p, franks, words, O, (unsigned char *)ctx->out.p,
                             ctx->sm_count, ctx->stream, (const int64_t *)ctx->wbounds.p, c));
      CK(cudaEventRecord(ctx->copy_ev[c], ctx->stream));
      CK(cudaStreamWaitEvent(ctx->copy, ctx->copy_ev[c], 0));
      if (r1 <= r0) continue;
      for (int k = 0; k < O.n_out; k++) {
        const size_t wd = dtype_size(O.o[k].dtype);
        const size_t at = (size_t)O.o[k].offset + (size_t)r0 * wd;
        CK(cudaMemcpyAsync((char *)R->buf.p + at, (const char *)ctx->out.p + at, (size_t)(r1 - r0) * wd,
                           cudaMemcpyDeviceToHost, ctx->copy));
        if (O.o[k].null_offset >= 0) {
          const size_t nat = (size_t)O.o[k].null_offset + (size_t)(r0 / 32) * 4;
          CK(cudaMemcpyAsync((char *)R->buf.p + nat, (const char *)ctx->out.p + nat, (size_t)((r1 - r0 + 31) / 32) * 4,
                             cudaMemcpyDeviceToHost, ctx->copy));
        }
      }
    }
    CK(cudaEventRecord(ctx->copy_ev[EMIT_CHUNKS], ctx->copy));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->copy_ev[EMIT_CHUNKS], 0));
  } else if (walk) {
    qm_scan_args a;
    fill_args(gt, a, (qm_status *)ctx->status.p);
    if (G > 0)
      CK(qm_launch_emit_walk(a, (const uint32_t *)ctx->fbits.p, (const uint64_t *)ctx->franks.p, rank_words(gt), O,
                             (unsigned char *)ctx->out.p, ctx->sm_count, ctx->stream));
  } else if (ranked && gt.small_rank) {
    if (G > 0)
      CK(qm_launch_emit_sorted(gt.table, ex.stride, (const uint32_t *)ctx->perm.p, (const uint64_t *)ctx->franks.p, G,
                               pl.key, ex.n_slots, O, (unsigned char *)ctx->out.p, ctx->sm_count, ctx->stream));
  } else if (ranked && G >= PERM_MIN_ROWS && ex.total_slots < ((int64_t)1 << 32)) {
    if ((rc = ensure(ctx, ctx->perm, sizeof(uint32_t) * (size_t)ex.total_slots))) {
      delete R;
      return rc;
    }
    CK(qm_launch_emit_perm(gt.table, ex.total_slots, ex.stride, pl.agg.acc[pl.agg.acc_count].word, first_word_o,
                           (const uint32_t *)ctx->fbits.p, (const uint64_t *)ctx->franks.p, rank_words(gt),
                           (uint32_t *)ctx->perm.p, G, pl.key, ex.n_slots, O, (unsigned char *)ctx->out.p,
                           ctx->sm_count, ctx->stream));
  } else if (ranked) {
    if (G > 0)
      CK(qm_launch_emit_ranked(gt.table, ex.total_slots, ex.stride, pl.agg.acc[pl.agg.acc_count].word, first_word_o,
                               (const uint32_t *)ctx->fbits.p, (const uint64_t *)ctx->franks.p, rank_words(gt),
                               pl.key, ex.n_slots, O,
                               (unsigned char *)ctx->out.p, ctx->sm_count, ctx->stream));
  } else {
    CK(qm_launch_emit(gt.table, ex.stride, slots, G, pl.key, ex.n_slots, O, (unsigned char *)ctx->out.p,
                      ctx->sm_count, ctx->stream));
  }
  if (G > 0) ctx->launches++;
  // post-aggregate ORDER BY / LIMIT / OFFSET: only the selected rows come back
  const void *res_dev = ctx->out.p;
  size_t res_bytes = off;
  if (pl.post) {
    qm_outspec O2;
    int64_t G2 = 0;
    size_t b2 = 0;
    if ((rc = post_aggregate(ctx, pl, O, G, O2, &G2, &b2))) {
      delete R;
      return rc;
    }
    O = O2;
    G = G2;
    res_dev = ctx->out2.p;
    res_bytes = b2;
  }
  if (!chunked) CK(cudaMemcpyAsync(R->buf.p, res_dev, res_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  cudaError_t se = cudaStreamSynchronize(ctx->stream);
  if (se != cudaSuccess) {
    delete R;
    return set_err(ctx, QM_ERR_CUDA, "finalize: %s", cudaGetErrorString(se));
  }
  float tail_ms = 0;
  cudaEventElapsedTime(&tail_ms, ctx->ev0, ctx->ev1);
  if (spec) {
    memcpy(spec, ctx->hstatus.p, sizeof(qm_status));
    take_scan_time(ctx, gt, spec->error == QM_DEV_OK);
    if (spec->error != QM_DEV_OK) {
      delete R;
      *out = nullptr;
      return QM_OK;
    }
    gt.selected = spec->rows_selected;
    G = (int64_t)*(uint64_t *)((char *)ctx->hstatus.p + 32);
  }

  R->n_rows = G;
  const uint8_t *h = (const uint8_t *)R->buf.p;
  for (int k = 0; k < O.n_out; k++) {
    qm_result::Col c;
    c.name = pl.meta[k].name;
    c.dtype = O.o[k].dtype;
    c.is_key = pl.meta[k].is_key;
    c.bytes = (size_t)G * dtype_size(c.dtype);
    c.data = h + O.o[k].offset;
    if (O.o[k].null_offset >= 0) {
      c.nulls = h + O.o[k].null_offset;
      const size_t nb = (size_t)((G + 7) / 8);
      for (size_t b = 0; b < nb && !c.has_nulls; b++) c.has_nulls = c.nulls[b] != 0;
    }
    R->cols.push_back(std::move(c));
  }
  R->stats.groups = G;
  R->stats.strategy = ex.strategy;
  R->stats.table_capacity = ilog2_ceil(std::max<int64_t>(ex.n_slots, 1));
  R->stats.retries = gt.retries;
  R->stats.rows_selected = (int64_t)gt.selected;
  R->stats.device_ms = (double)(scan_ms_so_far > tail_ms ? scan_ms_so_far : tail_ms);
  R->stats.scan_ms = gt.scan_ms;
  R->stats.launches = ctx->launches;
  *out = R;
  return QM_OK;
}

// Sizes the table for `est_groups` groups and allocates it (from ctx for a
// one-shot run, owned for a stream).
int setup_table(qm_ctx *ctx, GroupTable &gt, int64_t est_groups, int64_t direct_size, bool owned) {
  Plan &pl = gt.pl;
  Exec &ex = gt.ex;
  if (pl.key.mode == QK_NONE) {
    ex.n_slots = 1;
  } else if (pl.key.mode == QK_DIRECT) {
    ex.n_slots = direct_size;
  } else {
    int64_t want = std::max<int64_t>(1024, est_groups * 2 + est_groups / 8);
    ex.log2cap = ilog2_ceil(want);
    if (ex.log2cap > 31) ex.log2cap = 31;
    ex.n_slots = (int64_t)1 << ex.log2cap;
  }
  choose_layout(pl, est_groups, ex, ctx->tuning);
  size_t bytes = (size_t)ex.total_slots * ex.stride * 8;
  DevBuf &buf = owned ? gt.own : ctx->table;
  if (owned && !buf.p && ctx->agg_spare.bytes >= bytes) std::swap(buf, ctx->agg_spare);
  int rc = ensure(ctx, buf, bytes);
  if (rc) return rc;
  gt.table = (uint64_t *)buf.p;
  return init_table(ctx, gt);
}

int run_scan(qm_ctx *ctx, GroupTable &gt, int64_t n, const uint32_t *sel, bool timed = true, int bps_cap = 0) {
  qm_scan_args a;
  fill_args(gt, a, (qm_status *)ctx->status.p);
  a.n = n;
  a.sel = sel;
  a.row_offset = gt.rows_done;
  // staged filter columns are opt-in: measured slower than direct vector
  // loads at the occupancy their buffers allow
  int depth = ctx->tuning.stage_depth <= 0 ? 0 : ctx->tuning.stage_depth;
  if (depth > QM_STAGE_MAX_DEPTH) depth = QM_STAGE_MAX_DEPTH;
  bool staged = false;
  // per-warp copies pay for their set-up and fold only when every warp has
  // many tiles to aggregate
  if (a.priv && n < PRIV_MIN_ROWS) a.priv = 0;
  size_t smem = qm_scan_smem_bytes(gt.ex.local_slots, gt.ex.local_hash, gt.pl.agg.n_words, 0, 0, a.priv);
  if (!sel && !gt.zones && depth >= 2 && n >= (int64_t)QM_TILE_ROWS * 256) {
    for (; depth >= 2 && !staged; depth--) {
      if (!setup_staging(a.pred, a.stage, depth)) break;
      size_t sm = qm_scan_smem_bytes(gt.ex.local_slots, gt.ex.local_hash, gt.pl.agg.n_words, a.stage.tile_bytes, depth,
                                     a.priv);
      if (sm <= SMEM_LIMIT) {
        smem = sm;
        staged = true;
      }
    }
  }
  if (!staged) memset(&a.stage, 0, sizeof a.stage);
  int blocks = scan_blocks(ctx, smem, n, staged, bps_cap);
  if (timed) CK(cudaEventRecord(ctx->evs0, ctx->stream));
  CK(qm_launch_scan(a, blocks, smem, ctx->stream));
  if (timed) CK(cudaEventRecord(ctx->evs1, ctx->stream));
  if (n > 0) ctx->launches++;
  gt.scan_pending = true;
  return QM_OK;
}

// Partitioned aggregation (qm_part.cu, opt-in: qm_tuning.partitioned) for a
// grouped query whose table does not fit a block's shared memory and which
// selects many rows per group: survivors go to key partitions first and each
// partition is aggregated in shared memory instead of by per-row atomics on
// the group table.  Needs a selected fraction of at least PART_MIN_SEL
// (below it the scan, not the aggregation, dominates) and at least
// PART_MIN_ROWS_PER_GROUP selected rows per group.  Off by default: on the
// measured workloads the fused scan is faster (a 37M-row, 9,304-group query
// at 87 % selected: 1.46 ms against 1.20 ms; shared-memory aggregation of
// this shape runs at about 45 G rows/s, so counting, scattering and
// aggregating cannot beat the scan's L2 atomics).
constexpr size_t PART_SMEM = 96 * 1024;  // a partition's shared-memory table
// At most this many partitions: the scatter keeps one open write line per
// (partition, block), and beyond ~512 x 300 of them they no longer fit L2.
constexpr int PART_MAX = 512;
constexpr double PART_MIN_SEL = 0.25;
constexpr int64_t PART_MIN_ROWS_PER_GROUP = 4;
constexpr int64_t PART_MIN_ROWS = (int64_t)4 << 20;

struct PartPlan {
  qm_part_spec spec{};
  bool on = false;
};

int plan_partitioned(qm_ctx *ctx, qm_table *t, GroupTable &gt, int64_t est_groups, PartPlan &pp) {
  const int64_t n_rows = t->n_rows;
  pp.on = false;
  const Plan &pl = gt.pl;
  const Exec &ex = gt.ex;
  if (!ctx->tuning.partitioned || ctx->tuning.local_slots < 0 || pl.key.mode == QK_NONE || n_rows < PART_MIN_ROWS ||
      n_rows > 0xffffffffLL)
    return QM_OK;
  for (int c = 0; c < pl.agg.n_vcols; c++)
    if (pl.agg.vcol[c].flags & VF_FIXED) return QM_OK;
  if (pl.agg.n_vcols > QM_MAX_VCOLS - 2) return QM_OK;
  if (ex.local_slots > 0 && !ex.local_hash) return QM_OK;  // the whole direct table fits shared memory
  const int64_t groups = pl.key.mode == QK_DIRECT ? std::min<int64_t>(ex.n_slots, std::max<int64_t>(est_groups, 1))
                                                  : std::max<int64_t>(est_groups, 1);
  const int64_t slot_bytes = (int64_t)pl.agg.n_words * 8 + (pl.key.mode == QK_HASH ? 8 : 0);
  if (groups * slot_bytes <= (int64_t)PART_SMEM / 2) return QM_OK;  // fits the scan's block-local table
  int64_t sel = n_rows;
  if (has_filter(pl.pred)) {
    if (gt.sel_bound < 0) {
      int rc = table_sel_bound(ctx, t, pl.pred, &gt.sel_bound);
      if (rc) return rc;
    }
    sel = gt.sel_bound;
    if ((double)sel < PART_MIN_SEL * (double)n_rows) return QM_OK;
  }
  if (sel < PART_MIN_ROWS_PER_GROUP * groups) return QM_OK;
  qm_part_spec &ps = pp.spec;
  memset(&ps, 0, sizeof ps);
  ps.rec_words = (2 + pl.agg.n_vcols + 3) & ~3;  // whole 32-byte sectors
  ps.rec_cap = sel;
  int L = 1;
  while ((int64_t)(L * 2) * slot_bytes <= (int64_t)PART_SMEM) L *= 2;
  if (pl.key.mode == QK_DIRECT) {
    int shift = 0;
    while (((int64_t)1 << (shift + 1)) <= L) shift++;
    int64_t parts = (ex.n_slots + ((int64_t)1 << shift) - 1) >> shift;
    if (parts > PART_MAX) return QM_OK;
    ps.direct = 1;
    ps.shift = shift;
    ps.parts = (int)parts;
    ps.local_slots = 1 << shift;
  } else {
    int bits = 0;
    while (bits < 9 && ((int64_t)L / 4) * ((int64_t)1 << bits) < groups) bits++;
    if (((int64_t)L / 4) * ((int64_t)1 << bits) < groups) return QM_OK;  // too many keys per partition
    ps.direct = 0;
    ps.bits = bits;
    ps.parts = 1 << bits;
    ps.local_slots = L;
  }
  pp.on = true;
  return QM_OK;
}

// Runs the partitioned aggregation of n rows into gt's (initialised) table.
int run_partitioned(qm_ctx *ctx, GroupTable &gt, int64_t n, PartPlan &pp) {
  qm_scan_args a;
  fill_args(gt, a, (qm_status *)ctx->status.p);
  a.n = n;
  a.sel = nullptr;
  a.row_offset = gt.rows_done;
  a.priv = 0;
  memset(&a.stage, 0, sizeof a.stage);
  qm_part_spec &ps = pp.spec;
  ps.blocks = qm_part_scan_blocks(ctx->sm_count, ps.parts);
  const int64_t cells = (int64_t)(ps.parts + 1) * ps.blocks;
  int rc;
  if ((rc = ensure(ctx, ctx->part_counts, (size_t)cells * 4)) || (rc = ensure(ctx, ctx->part_offsets, (size_t)cells * 8)) ||
      (rc = ensure(ctx, ctx->part_bases, (size_t)(ps.parts + 2) * 8 + 64)) ||
      (rc = ensure(ctx, ctx->part_records, (size_t)std::max<int64_t>(ps.rec_cap, 1) * ps.rec_words * 8)))
    return rc;
  ps.counts = (uint32_t *)ctx->part_counts.p;
  ps.offsets = (uint64_t *)ctx->part_offsets.p;
  ps.bases = (uint64_t *)ctx->part_bases.p;
  ps.counter = (int *)((char *)ctx->part_bases.p + (size_t)(ps.parts + 2) * 8);
  ps.records = (uint64_t *)ctx->part_records.p;
  CK(cudaEventRecord(ctx->evs0, ctx->stream));
  CK(cudaMemsetAsync(ps.counter, 0, sizeof(int), ctx->stream));
  CK(qm_launch_part_scan(0, a, ps, ctx->stream));
  CK(qm_launch_part_offsets(ps, ctx->stream));
  CK(qm_launch_part_scan(1, a, ps, ctx->stream));
  CK(qm_launch_part_agg(a, ps, ctx->sm_count, ctx->stream));
  CK(cudaEventRecord(ctx->evs1, ctx->stream));
  ctx->launches += 5;
  gt.scan_pending = true;
  return QM_OK;
}

struct TableSource {  // a registered table's columns as the planner sees them
  ColEnv env;
};

int plan_query(qm_ctx *ctx, const qm_query *q, const ColEnv &env, Plan &pl) {
  if (!q) return set_err(ctx, QM_ERR_INVALID, "null query");
  std::vector<const DevCol *> touched;
  int64_t bpr = 0;
  int rc = build_pred(ctx, q, env, pl.pred, bpr, touched);
  if (rc) return rc;
  rc = build_agg(ctx, q, env, pl, touched);
  if (rc) return rc;
  pl.bytes_per_row = 0;
  for (auto *c : touched) pl.bytes_per_row += (int64_t)dtype_size(c->dtype);
  // post-aggregate ordering (src/operators.ts:3116-3128)
  pl.post = 0;
  pl.post_col = -1;
  if (q->offset < 0 || (q->has_limit && q->limit < 0))
    return set_err(ctx, QM_ERR_INVALID, "LIMIT and OFFSET are non-negative");
  pl.post_has_limit = q->has_limit ? 1 : 0;
  pl.post_limit = q->has_limit ? q->limit : 0;
  pl.post_offset = q->offset;
  pl.post_desc = q->order_desc ? 1 : 0;
  if (q->order_by) {
    for (int k = 0; k < (int)pl.meta.size(); k++)
      if (pl.meta[k].name == q->order_by) pl.post_col = k;
    pl.post = q->has_limit ? 3 : 2;
  } else if (q->has_limit || q->offset) {
    pl.post = 1;
  }
  return QM_OK;
}

}  // namespace


// ================================================================== C ABI

namespace {

// Zone maps of one column, computed on first use and kept on the column
// (like its min / max): per zone of QM_ZONE_ROWS rows the non-NULL (non-NaN)
// cells' min, max and count.
int column_zones(qm_ctx *ctx, DevCol &c, int64_t n) {
  if (c.has_zones) return QM_OK;
  const int64_t zones = (n + QM_ZONE_ROWS - 1) / QM_ZONE_ROWS;
  int rc = ensure(ctx, ctx->zstat, (size_t)std::max<int64_t>(zones, 1) * 24);
  if (rc) return rc;
  int64_t *d = (int64_t *)ctx->zstat.p;
  CK(qm_launch_zone_stats(c.data, c.dtype, c.nulls, n, d, d + zones, d + 2 * zones, ctx->stream));
  std::vector<int64_t> h((size_t)zones * 3);
  if (zones) CK(cudaMemcpyAsync(h.data(), d, (size_t)zones * 24, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  c.zmin.assign(h.begin(), h.begin() + zones);
  c.zmax.assign(h.begin() + zones, h.begin() + 2 * zones);
  c.zcount.assign(h.begin() + 2 * zones, h.end());
  c.has_zones = true;
  return QM_OK;
}

// Can term t reject every row of zone z?  A row passes t when its cell is
// NULL and t.null_pass, or when its value passes the test; the zone map
// bounds the values (NaN cells, which pass no range test, are outside it).
bool zone_rejects(const qm_term &t, const DevCol &c, int64_t z, int64_t zone_rows) {
  const bool isf = c.dtype == QM_F64 || c.dtype == QM_F32;
  if (t.kind == QT_TRUE)  // passes every non-NULL cell: rejects a zone of NULLs only
    return !t.null_pass && !isf && c.zcount[z] == 0;
  const int64_t cnt = c.zcount[z];
  const bool all_present = cnt == zone_rows;  // no NULL (nor NaN) cell
  if (t.null_pass && !all_present) return false;
  bool value_may_pass = cnt > 0;
  if (value_may_pass) {
    if (t.kind == QT_IRANGE && !isf) {
      value_may_pass = !(c.zmax[z] < t.lo || c.zmin[z] > t.hi);
    } else if (t.kind == QT_INRANGE && !isf) {
      value_may_pass = !(t.lo <= c.zmin[z] && c.zmax[z] <= t.hi);
    } else if (t.kind == QT_FRANGE && isf) {
      double mn, mx;
      memcpy(&mn, &c.zmin[z], 8);
      memcpy(&mx, &c.zmax[z], 8);
      value_may_pass = !(mx < t.f0 || mn > t.f1);
    } else if (t.kind == QT_FALSE) {
      value_may_pass = false;
    } else {
      return false;  // other tests: no bound from the zone map
    }
  }
  return !value_may_pass;
}

// Zones of table t that the plan's predicate may match (AND terms: one
// rejecting term rejects the zone; OR groups: every group must reject).
// Leaves gt.zones null when every zone stays.
int plan_zones(qm_ctx *ctx, qm_table *t, GroupTable &gt) {
  gt.zones = nullptr;
  gt.n_zone_tiles = 0;
  const qm_pred &P = gt.pl.pred;
  const int64_t n = t->n_rows;
  const int64_t nz = (n + QM_ZONE_ROWS - 1) / QM_ZONE_ROWS;
  const int nt = P.n_groups > 0 ? P.group_end[P.n_groups - 1] : P.n_and;
  if (nz < 4 || nt == 0) return QM_OK;
  std::vector<DevCol *> tc(nt, nullptr);
  bool any = false;
  for (int i = 0; i < nt; i++) {
    const qm_term &term = P.t[i];
    if (term.kind == QT_TRUE && term.null_pass) continue;
    for (auto &c : t->cols)
      if (c.data == term.data) tc[i] = &c;
    if (!tc[i]) continue;
    int rc = column_zones(ctx, *tc[i], n);
    if (rc) return rc;
    any = true;
  }
  if (!any) return QM_OK;
  std::vector<uint32_t> kept;
  kept.reserve(nz);
  for (int64_t z = 0; z < nz; z++) {
    const int64_t rows = std::min<int64_t>(QM_ZONE_ROWS, n - z * QM_ZONE_ROWS);
    auto rej = [&](int i) { return tc[i] && zone_rejects(P.t[i], *tc[i], z, rows); };
    bool skip = false;
    for (int i = 0; i < P.n_and && !skip; i++) skip = rej(i);
    if (!skip && P.n_groups > 0) {
      bool all = true;
      int b = P.n_and;
      for (int g = 0; g < P.n_groups && all; g++) {
        bool grp = false;
        for (int i = b; i < P.group_end[g] && !grp; i++) grp = rej(i);
        all = grp;
        b = P.group_end[g];
      }
      skip = all;
    }
    if (!skip) kept.push_back((uint32_t)z);
  }
  if ((int64_t)kept.size() == nz) return QM_OK;
  int rc = ensure(ctx, ctx->zones, std::max<size_t>(kept.size(), 1) * 4);
  if (rc) return rc;
  if (!kept.empty())
    CK(cudaMemcpyAsync(ctx->zones.p, kept.data(), kept.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  gt.zones = (const uint32_t *)ctx->zones.p;
  gt.n_zone_tiles = (int64_t)kept.size() * QM_ZONE_TILES;
  return QM_OK;
}

// Integer sums of int32 cells over a table of fewer than 2^32 rows stay
// within a signed 64-bit word (|sum| < 2^32 * 2^31), so the global table
// takes them with plain 64-bit atomic adds, which need no returned value.
void plan_narrow_sums(Plan &pl, int64_t n_rows) {
  if (n_rows >= ((int64_t)1 << 32)) return;
  qm_aggspec &A = pl.agg;
  for (int i = 0; i < A.n_accs; i++) {
    qm_acc &ac = A.acc[i];
    if (ac.kind != QA_ISUM || ac.wide) continue;
    ac.narrow = 1;
    for (int c = 0; c < A.n_vcols; c++)
      if ((A.vcol[c].flags & VF_SUM) && A.vcol[c].w_sum == ac.word) A.vcol[c].flags |= VF_NARROW;
    for (int k = 0; k < pl.outs.n_out; k++) {
      qm_out &o = pl.outs.o[k];
      if ((o.kind == QO_SUM_I2F || o.kind == QO_AVG_I2F) && o.word == ac.word) o.narrow = 1;
    }
  }
}

// A dense (direct) group table larger than this is updated in key-range
// passes, each pass's slots staying in L2: the scan re-reads the key column
// once per pass, but every atomic update then hits L2 instead of DRAM.
#ifndef QM_L2_TABLE_MB
#define QM_L2_TABLE_MB 64
#endif
constexpr int64_t L2_TABLE_BUDGET = (int64_t)QM_L2_TABLE_MB << 20;

// Key-range passes for a direct-indexed table query (1: a single scan).
constexpr int KEY_RANGE_BLOCKS_PER_SM = 1;
int key_range_passes(const GroupTable &gt, int64_t n_rows, int64_t sel_bound) {
  const Plan &pl = gt.pl;
  if (pl.key.mode != QK_DIRECT || pl.key.n_cols != 1 || pl.key.pack != QP_RAW) return 1;
  if (pl.pred.n_and + (pl.pred.n_groups > 0 ? pl.pred.group_end[pl.pred.n_groups - 1] - pl.pred.n_and : 0) >=
      QM_MAX_TERMS)
    return 1;
  const int64_t bytes = gt.ex.total_slots * gt.ex.stride * 8;
  if (bytes <= L2_TABLE_BUDGET) return 1;
  // worth it when rows outnumber slots (dense updates); a selective filter
  // leaves few atomics to save
  const int64_t rows = sel_bound >= 0 ? sel_bound : n_rows;
  if (rows < gt.ex.n_slots) return 1;
  return (int)std::min<int64_t>(64, (bytes + L2_TABLE_BUDGET - 1) / L2_TABLE_BUDGET);
}

// The predicate with an extra AND term: key in [lo, hi] (NULL keys pass in
// one chosen pass only, so each row is aggregated exactly once).
qm_pred with_key_range(const qm_pred &P, const qm_keyspec &K, int64_t lo, int64_t hi, bool nulls_pass) {
  qm_pred q = P;
  const int nt = P.n_groups > 0 ? P.group_end[P.n_groups - 1] : P.n_and;
  for (int i = nt; i > P.n_and; i--) q.t[i] = P.t[i - 1];
  for (int g = 0; g < P.n_groups; g++) q.group_end[g] = P.group_end[g] + 1;
  qm_term &t = q.t[P.n_and];
  memset(&t, 0, sizeof t);
  t.data = K.data[0];
  t.nulls = K.nulls[0];
  t.dtype = K.dtype[0];
  t.kind = QT_IRANGE;
  t.null_pass = nulls_pass ? 1 : 0;
  t.sidx = -1;
  t.lo = lo;
  t.hi = hi;
  q.n_and = P.n_and + 1;
  return q;
}

// Plan `q` over registered table `t`: lower it, pack its keys, pick the
// key mode (direct when the key range from column statistics is dense, else
// hash) and estimate the group count (HyperLogLog, cached per column).
int plan_table_query(qm_ctx *ctx, qm_table *t, const qm_query *q, GroupTable &gt, int64_t &est,
                     int64_t &direct_size) {
  ColEnv env;
  for (auto &c : t->cols) env.views.push_back({&c, t->n_rows});
  int rc = plan_query(ctx, q, env, gt.pl);
  if (rc) return rc;
  Plan &pl = gt.pl;
  est = 1;
  direct_size = 0;
  uint64_t space = 0;
  if ((rc = plan_key_packing(ctx, pl, t->n_rows, true, &space))) return rc;
  if ((rc = plan_split_sums(ctx, pl, t->n_rows, (q->flags & QM_FLAG_DETERMINISTIC) != 0))) return rc;
  plan_narrow_sums(pl, t->n_rows);
  if (pl.key.n_cols == 0) {
    pl.key.mode = QK_NONE;
  } else {
    const ColView *kv = env.find(q->group_by[0]);
    DevCol &kc = *const_cast<DevCol *>(kv->col);
    bool direct = false;
    if (pl.key.pack == QP_DIGITS) {
      if (space <= (1ULL << 25) && (int64_t)space <= std::max<int64_t>(4 * t->n_rows, 1 << 16)) {
        direct = true;
        direct_size = (int64_t)space;
        pl.key.base = 0;
      }
    } else if (pl.key.n_cols == 1 && is_int(kc.dtype)) {
      if ((rc = column_minmax(ctx, kc, t->n_rows))) return rc;
      if (kc.mx >= kc.mn) {
        unsigned long long range = (unsigned long long)kc.mx - (unsigned long long)kc.mn + 1ULL;
        if (range != 0 && range <= (1ULL << 25) && (int64_t)range <= std::max<int64_t>(4 * t->n_rows, 1 << 16)) {
          direct = true;
          direct_size = (int64_t)range;
          pl.key.base = kc.mn;
        }
      } else {
        direct = true;  // no non-null key: only the NULL slot is used
        direct_size = 1;
        pl.key.base = 0;
      }
    }
    const bool single = pl.key.n_cols == 1;
    // a wide dense range that a selective filter leaves mostly empty: a hash
    // table sized by the selected rows is smaller to clear and to compact
    int64_t sel_bound = -1;  // sampled bound on selected rows, when taken
    if (direct && direct_size > (1 << 20) && t->n_rows >= 4 * (int64_t)SEL_SAMPLES && has_filter(pl.pred)) {
      if ((rc = table_sel_bound(ctx, t, pl.pred, &sel_bound))) return rc;
      if (sel_bound * 4 < direct_size) direct = false;
    }
    if (direct) {
      pl.key.mode = QK_DIRECT;
      est = direct_size;
      if (direct_size > (1 << 16)) {
        double e = 0;
        if (single && kc.has_hll) {
          e = kc.hll;
        } else {
          qm_keyspec K = pl.key;
          K.mode = QK_HASH;
          if ((rc = estimate_groups(ctx, K, t->n_rows, &e))) return rc;
          if (single) {
            kc.hll = e;
            kc.has_hll = true;
          }
        }
        est = std::min<int64_t>(est, (int64_t)(e * 1.05) + 16);
      }
    } else {
      pl.key.mode = QK_HASH;
      if (single && kc.has_hll) {
        est = (int64_t)(kc.hll * 1.05) + 16;
      } else {
        qm_keyspec K = pl.key;
        double e;
        if ((rc = estimate_groups(ctx, K, t->n_rows, &e))) return rc;
        est = (int64_t)(e * 1.05) + 16;
        if (pl.key.n_cols == 1) {
          kc.hll = e;
          kc.has_hll = true;
        }
      }
      est = std::min<int64_t>(est, std::max<int64_t>(t->n_rows, 1));
      // a filtered query has at most as many groups as selected rows
      if (est > 65536 && t->n_rows >= 4 * (int64_t)SEL_SAMPLES && has_filter(pl.pred)) {
        if (sel_bound < 0 && (rc = table_sel_bound(ctx, t, pl.pred, &sel_bound))) return rc;
        est = std::min(est, sel_bound);
      }
    }
    gt.sel_bound = sel_bound;
  }
  return QM_OK;
}

}  // namespace

extern "C" {



const char *qm_version(void) { return "querymode-b200 0.1 (sm_100a)"; }

int qm_ctx_create(int32_t device, qm_ctx **out) {
  if (!out) return QM_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return QM_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return QM_ERR_INVALID;
  qm_ctx *ctx = new qm_ctx();
  ctx->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  ctx->stream = ctx->own_stream;
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evs0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evs1);
  cudaDeviceProp prop;
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return QM_ERR_CUDA;
  }
  ctx->sm_count = prop.multiProcessorCount;
  ctx->hbm_bytes = (int64_t)prop.totalGlobalMem;
  {
    // stream-ordered allocations (batch buffers) stay in the device's pool
    // when freed, for the next batch of that size, instead of going back to
    // the driver at every synchronisation; qm_ctx_trim hands them back
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  if (ensure(ctx, ctx->status, sizeof(qm_status))) {
    delete ctx;
    return QM_ERR_OOM;
  }
  *out = ctx;
  return QM_OK;
}

int qm_ctx_destroy(qm_ctx *ctx) {
  if (!ctx) return QM_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  DevBuf *bufs[] = {&ctx->table, &ctx->status, &ctx->keys, &ctx->slots, &ctx->keys2, &ctx->slots2,
                    &ctx->sort_temp, &ctx->counter, &ctx->out, &ctx->hll, &ctx->masks, &ctx->counts,
                    &ctx->offsets, &ctx->sel_out, &ctx->sel_in, &ctx->agg_spare, &ctx->fbits, &ctx->fcounts,
                    &ctx->franks, &ctx->post_last, &ctx->post_hi, &ctx->post_lo, &ctx->post_idx,
                    &ctx->post_idx2, &ctx->post_k1, &ctx->post_k2, &ctx->post_l1, &ctx->post_l2,
                    &ctx->post_temp, &ctx->out2, &ctx->zstat, &ctx->zones, &ctx->ustat, &ctx->perm,
                    &ctx->wbounds, &ctx->part_counts, &ctx->part_offsets, &ctx->part_bases, &ctx->part_records};
  for (DevBuf *b : bufs) release(*b);
  for (auto &b : ctx->staged) release(b);
  ctx->dpool.trim();
  if (ctx->hout.p) cudaFreeHost(ctx->hout.p);
  if (ctx->hstatus.p) cudaFreeHost(ctx->hstatus.p);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->evs0) cudaEventDestroy(ctx->evs0);
  if (ctx->evs1) cudaEventDestroy(ctx->evs1);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  if (ctx->copy) cudaStreamDestroy(ctx->copy);
  for (cudaEvent_t e : ctx->copy_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->aux_ev) cudaEventDestroy(ctx->aux_ev);
  delete ctx;
  return QM_OK;
}

int qm_ctx_trim(qm_ctx *ctx, int64_t *released) {
  if (!ctx) return QM_ERR_INVALID;
  cudaSetDevice(ctx->device);
  size_t bytes;
  {
    std::lock_guard<std::mutex> lk(ctx->dpool.mu);
    bytes = ctx->dpool.cached;
  }
  ctx->dpool.trim();
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(pool, 0);
  }
  cudaGetLastError();
  if (released) *released = (int64_t)bytes;
  return QM_OK;
}

int qm_ctx_set_tuning(qm_ctx *ctx, const qm_tuning *t) {
  if (!ctx) return QM_ERR_INVALID;
  if (!t) {
    ctx->tuning = qm_tuning{0, -1, 0, 0, 0, 0};
    return QM_OK;
  }
  if (t->local_slots > 0 && (t->local_slots & (t->local_slots - 1)))
    return set_err(ctx, QM_ERR_INVALID, "local_slots must be a power of two");
  if (t->local_slots > (1 << 14)) return set_err(ctx, QM_ERR_INVALID, "local_slots too large");
  ctx->tuning = *t;
  return QM_OK;
}

int qm_ctx_set_stream(qm_ctx *ctx, void *stream) {
  if (!ctx) return QM_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return QM_OK;
}

const char *qm_ctx_last_error(const qm_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int qm_ctx_device_info(const qm_ctx *ctx, int32_t *sm_count, int64_t *hbm_bytes) {
  if (!ctx) return QM_ERR_INVALID;
  if (sm_count) *sm_count = ctx->sm_count;
  if (hbm_bytes) *hbm_bytes = ctx->hbm_bytes;
  return QM_OK;
}

// Tables of at least this many rows get their column statistics at upload.
constexpr int64_t EAGER_STATS_ROWS = (int64_t)4 << 20;

int qm_table_create(qm_ctx *ctx, int64_t n_rows, int32_t n_cols, const qm_column *cols, qm_table **out) {
  if (!ctx || !out || n_rows < 0 || n_cols < 0 || (n_cols > 0 && !cols))
    return set_err(ctx, QM_ERR_INVALID, "qm_table_create: bad arguments");
  if (n_rows > 0xffffffffLL)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "tables are limited to 2^32-1 rows (QMCB rowCount is u32)");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  qm_table *t = new qm_table();
  t->ctx = ctx;
  t->n_rows = n_rows;
  // The planner's column statistics (min / max of integer columns, max |x|
  // of float columns, zone maps) of host-uploaded columns are computed on a
  // side stream behind each column's copy, while the next columns cross the
  // host link, instead of on the first query with a synchronise each.
  const int64_t zones = (n_rows + QM_ZONE_ROWS - 1) / QM_ZONE_ROWS;
  const size_t per = 32 + (size_t)zones * 24;
  bool eager = n_rows >= EAGER_STATS_ROWS;
  HostBuf hs;
  if (eager) {
    if ((!ctx->aux && cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess) ||
        (!ctx->aux_ev && cudaEventCreateWithFlags(&ctx->aux_ev, cudaEventDisableTiming) != cudaSuccess) ||
        ensure(ctx, ctx->ustat, per * std::max(n_cols, 1)) != QM_OK || !ctx->pool->acquire(per * std::max(n_cols, 1), hs)) {
      cudaGetLastError();
      eager = false;  // the statistics stay lazy
    }
  }
  std::vector<char> staged((size_t)n_cols, 0);
  auto fail = [&](int rc) {
    if (eager) cudaStreamSynchronize(ctx->aux);
    ctx->pool->release(hs);
    qm_table_destroy(t);
    return rc;
  };
  for (int i = 0; i < n_cols; i++) {
    for (auto &c : t->cols)
      if (c.name == cols[i].name) return fail(set_err(ctx, QM_ERR_INVALID, "duplicate column %s", cols[i].name));
    DevCol c;
    int rc = make_col(ctx, n_rows, cols[i], c);
    if (rc) {
      free_col(ctx, c);
      return fail(rc);
    }
    t->cols.push_back(c);
    if (eager && !cols[i].on_device) {
      uint8_t *d = (uint8_t *)ctx->ustat.p + per * i;
      int64_t *z = (int64_t *)(d + 32);
      cudaError_t e = cudaEventRecord(ctx->aux_ev, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->aux, ctx->aux_ev, 0);
      if (e == cudaSuccess)
        e = is_int(c.dtype) ? qm_launch_minmax(c.data, c.dtype, c.nulls, n_rows, (long long *)d, ctx->sm_count, ctx->aux)
                            : qm_launch_maxabs(c.data, c.dtype, c.nulls, n_rows, (unsigned long long *)(d + 16),
                                               ctx->sm_count, ctx->aux);
      if (e == cudaSuccess) e = qm_launch_zone_stats(c.data, c.dtype, c.nulls, n_rows, z, z + zones, z + 2 * zones, ctx->aux);
      if (e == cudaSuccess) e = cudaMemcpyAsync((uint8_t *)hs.p + per * i, d, per, cudaMemcpyDeviceToHost, ctx->aux);
      if (e != cudaSuccess) return fail(set_err(ctx, QM_ERR_CUDA, "column statistics: %s", cudaGetErrorString(e)));
      staged[i] = 1;
    }
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && eager) e = cudaStreamSynchronize(ctx->aux);
  if (e != cudaSuccess) return fail(set_err(ctx, QM_ERR_CUDA, "upload: %s", cudaGetErrorString(e)));
  for (int i = 0; i < n_cols; i++) {
    if (!staged[i]) continue;
    DevCol &c = t->cols[i];
    const uint8_t *h = (const uint8_t *)hs.p + per * i;
    if (is_int(c.dtype)) {
      memcpy(&c.mn, h, 8);
      memcpy(&c.mx, h + 8, 8);
      c.has_minmax = true;
    } else {
      memcpy(&c.maxabs, h + 16, 8);
      c.has_maxabs = true;
    }
    const int64_t *z = (const int64_t *)(h + 32);
    c.zmin.assign(z, z + zones);
    c.zmax.assign(z + zones, z + 2 * zones);
    c.zcount.assign(z + 2 * zones, z + 3 * zones);
    c.has_zones = true;
  }
  ctx->pool->release(hs);
  *out = t;
  return QM_OK;
}

int qm_table_from_qmcb(qm_ctx *ctx, const uint8_t *buf, size_t len, qm_table **out) {
  if (!ctx || !buf || !out) return set_err(ctx, QM_ERR_INVALID, "qm_table_from_qmcb: bad arguments");
  // decodeColumnarBatch layout (src/columnar.ts:438-516)
  if (len < 10) return set_err(ctx, QM_ERR_INVALID, "QMCB buffer shorter than its header");
  uint32_t magic, rows;
  uint16_t ncol;
  memcpy(&magic, buf, 4);
  memcpy(&rows, buf + 4, 4);
  memcpy(&ncol, buf + 8, 2);
  if (magic != 0x42434D51u) return set_err(ctx, QM_ERR_INVALID, "bad QMCB magic");
  struct D {
    std::string name;
    int dtype;
    bool nulls;
  };
  std::vector<D> descs;
  size_t pos = 10;
  for (int c = 0; c < ncol; c++) {
    if (pos + 2 > len) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB descriptor");
    uint16_t nl;
    memcpy(&nl, buf + pos, 2);
    pos += 2;
    if (pos + nl + 2 > len) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB descriptor");
    D d;
    d.name.assign((const char *)buf + pos, nl);
    pos += nl;
    d.dtype = buf[pos++];
    d.nulls = buf[pos++] != 0;
    descs.push_back(d);
  }
  std::vector<qm_column> cols;
  std::vector<std::string> names;
  names.reserve(descs.size());
  for (auto &d : descs) {
    const uint8_t *nb = nullptr;
    if (d.nulls) {
      size_t nbl = ((size_t)rows + 7) / 8;
      if (pos + nbl > len) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB null bitmap");
      nb = buf + pos;
      pos += nbl;
    }
    size_t sz = 0;
    switch (d.dtype) {
      case QM_F64: case QM_I64: sz = (size_t)rows * 8; break;
      case QM_I32: case QM_F32: sz = (size_t)rows * 4; break;
      case 2: {  // UTF8: total length, offsets, bytes
        if (pos + 4 > len) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB utf8 column");
        uint32_t tl;
        memcpy(&tl, buf + pos, 4);
        sz = 4 + ((size_t)rows + 1) * 4 + tl;
        break;
      }
      case 3: sz = ((size_t)rows + 7) / 8; break;  // BOOL
      case 4: {                                     // F32VEC: dim, data
        if (pos + 4 > len) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB vector column");
        uint32_t dim;
        memcpy(&dim, buf + pos, 4);
        // rows x dim x 4 can pass 2^64: a column larger than the buffer is truncated
        if (rows && dim > (len / 4) / rows) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB vector column");
        sz = 4 + (size_t)rows * dim * 4;
        break;
      }
      default: sz = 0;
    }
    if (pos > len || sz > len - pos) return set_err(ctx, QM_ERR_INVALID, "truncated QMCB column %s", d.name.c_str());
    if (valid_dtype(d.dtype)) {
      names.push_back(d.name);
      qm_column c;
      c.name = names.back().c_str();
      c.dtype = d.dtype;
      c.on_device = 0;
      c.data = buf + pos;
      c.null_bitmap = nb;
      cols.push_back(c);
    }
    pos += sz;
  }
  return qm_table_create(ctx, (int64_t)rows, (int32_t)cols.size(), cols.data(), out);
}

int qm_table_destroy(qm_table *t) {
  if (!t) return QM_OK;
  if (t->ctx) cudaSetDevice(t->ctx->device);
  if (t->ctx) cudaStreamSynchronize(t->ctx->stream);
  for (auto &c : t->cols) free_col(t->ctx, c);
  delete t;
  return QM_OK;
}

int qm_table_num_rows(const qm_table *t, int64_t *out) {
  if (!t || !out) return QM_ERR_INVALID;
  *out = t->n_rows;
  return QM_OK;
}

int qm_table_num_columns(const qm_table *t, int32_t *out) {
  if (!t || !out) return QM_ERR_INVALID;
  *out = (int32_t)t->cols.size();
  return QM_OK;
}

int qm_table_column(const qm_table *t, int32_t column, const char **name, int32_t *dtype) {
  if (!t || column < 0 || column >= (int32_t)t->cols.size()) return QM_ERR_INVALID;
  if (name) *name = t->cols[column].name.c_str();
  if (dtype) *dtype = t->cols[column].dtype;
  return QM_OK;
}

int qm_query_run(qm_ctx *ctx, const qm_table *table, const qm_query *q, qm_result **out) {
  if (!ctx || !table || !q || !out) return set_err(ctx, QM_ERR_INVALID, "qm_query_run: bad arguments");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  qm_table *t = const_cast<qm_table *>(table);
  ctx->launches = 0;
  GroupTable gt;
  int64_t est = 1, direct_size = 0;
  int rc = plan_table_query(ctx, t, q, gt, est, direct_size);
  if (rc) return rc;
  if ((rc = plan_zones(ctx, t, gt))) return rc;
  Plan &pl = gt.pl;
  gt.rows_done = 0;
  int64_t groups = -1;
  for (int attempt = 0;; attempt++) {
    gt.rows_done = 0;  // every attempt scans the table from its first row
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if ((rc = setup_table(ctx, gt, est, direct_size, false))) return rc;
    PartPlan pp;
    if ((rc = plan_partitioned(ctx, t, gt, est, pp))) return rc;
    if (pp.on && attempt > 0) pp.spec.rec_cap = t->n_rows;  // a re-run after an overflow: room for every row
    const int passes = pp.on ? 1 : key_range_passes(gt, t->n_rows, gt.sel_bound);
    if (pp.on) {
      if ((rc = run_partitioned(ctx, gt, t->n_rows, pp))) return rc;
      gt.ex.strategy = 3;
    } else if (passes <= 1) {
      if ((rc = run_scan(ctx, gt, t->n_rows, nullptr))) return rc;
    } else {
      const qm_pred base = pl.pred;
      const int64_t span = (gt.ex.n_slots + passes - 1) / passes;
      CK(cudaEventRecord(ctx->evs0, ctx->stream));
      for (int p = 0; p < passes; p++) {
        const int64_t lo = pl.key.base + p * span;
        const int64_t hi = std::min<int64_t>(pl.key.base + gt.ex.n_slots - 1, lo + span - 1);
        pl.pred = with_key_range(base, pl.key, lo, hi, p == 0);
        // one block per SM: fewer warps in flight keep more of the pass's
        // slots in L2 (200M rows x 16.7M groups: 9.87 -> 9.35 ms)
        rc = run_scan(ctx, gt, t->n_rows, nullptr, false, KEY_RANGE_BLOCKS_PER_SM);
        pl.pred = base;
        if (rc) return rc;
      }
      CK(cudaEventRecord(ctx->evs1, ctx->stream));
      gt.scan_pending = true;
    }
    // rank the groups before reading the status: one synchronize for both
    // (an overflowed table's ranking is discarded with it)
    gt.rows_done = t->n_rows;
    const bool ranked = ranked_finish(gt);
    if (ranked && (rc = launch_rank(ctx, gt))) return rc;
    qm_status st;
    qm_outspec Ocap = pl.outs;
    // a dense direct-indexed table (its groups fill most slots) costs no more
    // to copy laid out for every slot than for its groups
    const bool dense = pl.key.mode == QK_DIRECT && est * 4 >= gt.ex.total_slots * 3;
    if (ranked && !pl.post && (dense || result_layout(pl, Ocap, gt.ex.total_slots) <= SPEC_RESULT_BYTES)) {
      // small or dense result: emitted and copied with the status, one synchronise
      CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->status.p, sizeof(qm_status), cudaMemcpyDeviceToHost, ctx->stream));
      if ((rc = finish_table(ctx, gt, out, 0.f, -1, &st, true))) return rc;
      if (*out) {
        (*out)->stats.rows_scanned = t->n_rows;
        (*out)->stats.bytes_scanned = pl.bytes_per_row * t->n_rows;
        return QM_OK;
      }
    } else {
      if ((rc = read_status(ctx, &st))) return rc;
      take_scan_time(ctx, gt, st.error == QM_DEV_OK);
      if (st.error == QM_DEV_OK) {
        gt.selected = st.rows_selected;
        if (ranked) groups = (int64_t)*(uint64_t *)((char *)ctx->hstatus.p + 32);
        break;
      }
    }
    if (attempt >= 4) return set_err(ctx, QM_ERR_CUDA, "group table overflow after %d regrowths", attempt);
    gt.retries++;
    if (st.error == QM_DEV_STALE) {
      // a fixed-point SUM cell beyond its column's cached range: the column
      // changed since; take its statistics again and re-run
      for (int c = 0; c < pl.agg.n_vcols; c++)
        if (pl.vcolsrc[c]) const_cast<DevCol *>(pl.vcolsrc[c])->has_maxabs = false;
      if ((rc = plan_split_sums(ctx, pl, t->n_rows, true))) return rc;
      continue;
    }
    if (st.error == QM_DEV_RANGE || pl.key.mode == QK_DIRECT) {
      pl.key.mode = QK_HASH;
    }
    est = std::max<int64_t>(est * 4, (int64_t)st.groups_inserted * 2);
  }
  gt.rows_done = t->n_rows;
  rc = finish_table(ctx, gt, out, 0.f, groups, nullptr, true);
  if (rc) return rc;
  (*out)->stats.rows_scanned = t->n_rows;
  (*out)->stats.bytes_scanned = pl.bytes_per_row * t->n_rows;
  return QM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ streaming
struct qm_agg {
  qm_ctx *ctx = nullptr;
  std::vector<std::string> strs;  // owned copies of every name in the query
  std::vector<qm_filter> filters, or_filters;
  std::vector<int32_t> or_sizes;
  std::vector<const char *> group_by;
  std::vector<qm_aggregate> aggs;
  qm_query q{};
  GroupTable gt;
  bool planned = false;
  std::vector<std::pair<std::string, int>> schema;
  double device_ms = 0;
  bool failed = false;
};

namespace {

// Stage one batch's columns on the device: host columns are copied into
// grow-only per-column buffers of the context, null bitmaps into word-padded
// buffers.  Views point at the staged copies.
int stage_batch(qm_ctx *ctx, int64_t n, int32_t n_cols, const qm_column *cols, std::vector<DevCol> &out) {
  out.clear();
  if ((int)ctx->staged.size() < 2 * n_cols) ctx->staged.resize(2 * n_cols);
  for (int i = 0; i < n_cols; i++) {
    const qm_column &c = cols[i];
    if (!c.name) return set_err(ctx, QM_ERR_INVALID, "column without a name");
    if (!valid_dtype(c.dtype)) return set_err(ctx, QM_ERR_UNSUPPORTED, "column %s: dtype %d is not numeric", c.name, c.dtype);
    if (n > 0 && !c.data) return set_err(ctx, QM_ERR_INVALID, "column %s: no data", c.name);
    DevCol d;
    d.name = c.name;
    d.dtype = c.dtype;
    const size_t bytes = (size_t)n * dtype_size(c.dtype);
    if (c.on_device) {
      d.data = const_cast<void *>(c.data);
    } else {
      int rc = ensure(ctx, ctx->staged[2 * i], bytes + 16);
      if (rc) return rc;
      if (bytes) CK(cudaMemcpyAsync(ctx->staged[2 * i].p, c.data, bytes, cudaMemcpyHostToDevice, ctx->stream));
      d.data = ctx->staged[2 * i].p;
    }
    if (c.null_bitmap) {
      const size_t words = (size_t)((n + 31) / 32) + 1;
      int rc = ensure(ctx, ctx->staged[2 * i + 1], words * 4);
      if (rc) return rc;
      CK(cudaMemsetAsync(ctx->staged[2 * i + 1].p, 0, words * 4, ctx->stream));
      if (n > 0)
        CK(cudaMemcpyAsync(ctx->staged[2 * i + 1].p, c.null_bitmap, (size_t)((n + 7) / 8),
                           c.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
      d.nulls = (uint32_t *)ctx->staged[2 * i + 1].p;
    }
    out.push_back(d);
  }
  return QM_OK;
}

int stage_selection(qm_ctx *ctx, const uint32_t *sel, int64_t n_sel, const uint32_t **dsel) {
  *dsel = nullptr;
  if (!sel) return QM_OK;
  int rc = ensure(ctx, ctx->sel_in, (size_t)n_sel * 4 + 16);
  if (rc) return rc;
  cudaPointerAttributes at;
  bool on_dev = cudaPointerGetAttributes(&at, sel) == cudaSuccess && at.type == cudaMemoryTypeDevice;
  cudaGetLastError();
  if (on_dev) {
    *dsel = sel;
    return QM_OK;
  }
  if (n_sel) CK(cudaMemcpyAsync(ctx->sel_in.p, sel, (size_t)n_sel * 4, cudaMemcpyHostToDevice, ctx->stream));
  *dsel = (const uint32_t *)ctx->sel_in.p;
  return QM_OK;
}

// Grow a streaming hash table so that `upper` groups keep the load <= ~0.5.
int grow_table(qm_ctx *ctx, GroupTable &gt, int64_t upper) {
  Exec &ex = gt.ex;
  if (gt.pl.key.mode != QK_HASH || upper * 2 + upper / 8 <= ex.n_slots) return QM_OK;
  Exec nx = ex;
  nx.log2cap = ilog2_ceil(std::max<int64_t>(1024, upper * 2 + upper / 8));
  if (nx.log2cap > 31) return set_err(ctx, QM_ERR_OOM, "group table would exceed 2^31 slots");
  nx.n_slots = (int64_t)1 << nx.log2cap;
  nx.total_slots = nx.n_slots + 2;
  DevBuf nb;
  int rc = ensure(ctx, nb, (size_t)nx.total_slots * nx.stride * 8);
  if (rc) return rc;
  GroupTable tmp;
  tmp.pl = gt.pl;
  tmp.ex = nx;
  tmp.table = (uint64_t *)nb.p;
  if ((rc = init_table(ctx, tmp))) {
    release(nb);
    return rc;
  }
  CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
  CK(qm_launch_rehash(gt.table, ex.n_slots, ex.stride, gt.pl.agg.acc[gt.pl.agg.acc_count].word, tmp.table,
                      nx.log2cap, (qm_status *)ctx->status.p, ctx->sm_count, ctx->stream));
  // the two reserved slots (sentinel-valued key, NULL key) move as they are
  CK(cudaMemcpyAsync(tmp.table + nx.n_slots * nx.stride, gt.table + ex.n_slots * ex.stride,
                     (size_t)2 * ex.stride * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  qm_status st;
  if ((rc = read_status(ctx, &st))) {
    release(nb);
    return rc;
  }
  if (st.error) {
    release(nb);
    return set_err(ctx, QM_ERR_CUDA, "rehash overflow");
  }
  release(gt.own);
  gt.own = nb;
  gt.table = tmp.table;
  // local-table choice may change with the new size
  choose_layout(gt.pl, upper, nx, ctx->tuning);
  gt.ex = nx;
  return QM_OK;
}

// Distinct-key estimate of a streamed batch: the key column's cached
// HyperLogLog when it has one (a registered table's column), else a sketch
// of this batch.
int key_estimate(qm_ctx *ctx, const Plan &pl, int64_t n_rows, double *e) {
  if (pl.key.n_cols == 1 && pl.keycols[0]) {
    DevCol &kc = *const_cast<DevCol *>(pl.keycols[0]);
    if (kc.has_hll) {
      *e = kc.hll;
      return QM_OK;
    }
    int rc = estimate_groups(ctx, pl.key, n_rows, e);
    if (!rc) {
      kc.hll = *e;
      kc.has_hll = true;
    }
    return rc;
  }
  return estimate_groups(ctx, pl.key, n_rows, e);
}

// One pushed batch (columns in env) through the aggregation's table.
int agg_push_env(qm_agg *a, const ColEnv &env, int64_t n_rows, const uint32_t *dsel, int64_t n_elems) {
  qm_ctx *ctx = a->ctx;
  int rc;
  GroupTable &gt = a->gt;
  Plan pl;
  if ((rc = plan_query(ctx, &a->q, env, pl))) return rc;
  uint64_t space = 0;
  if ((rc = plan_key_packing(ctx, pl, n_rows, false, &space))) return rc;
  pl.key.mode = pl.key.n_cols == 0 ? QK_NONE : QK_HASH;
  if (!a->planned) {
    gt.pl = pl;
    int64_t est = 1;
    if (pl.key.mode == QK_HASH) {
      est = n_elems;
      if (n_elems > (1 << 16)) {
        double e;
        if ((rc = key_estimate(ctx, pl, n_rows, &e))) return rc;
        est = std::min<int64_t>(est, (int64_t)(e * 1.1) + 1024);
      }
    }
    if ((rc = setup_table(ctx, gt, std::max<int64_t>(est, 1), 0, true))) return rc;
    a->planned = true;
  } else {
    // same structure, this batch's column pointers
    pl.key.base = gt.pl.key.base;
    gt.pl.pred = pl.pred;
    gt.pl.agg = pl.agg;
    memcpy(gt.pl.key.data, pl.key.data, sizeof pl.key.data);
    memcpy(gt.pl.key.nulls, pl.key.nulls, sizeof pl.key.nulls);
    if (gt.pl.key.mode == QK_HASH) {
      int64_t add = n_elems;
      if (n_elems > (1 << 16)) {
        double e;
        if ((rc = key_estimate(ctx, pl, n_rows, &e))) return rc;
        add = std::min<int64_t>(add, (int64_t)(e * 1.1) + 1024);
      }
      if ((rc = grow_table(ctx, gt, gt.groups_upper + add))) return rc;
    }
  }
  CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if ((rc = run_scan(ctx, gt, n_elems, dsel))) return rc;
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  qm_status st;
  if ((rc = read_status(ctx, &st))) return rc;
  take_scan_time(ctx, gt, true);
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  a->device_ms += ms;
  if (st.error) {
    a->failed = true;
    return set_err(ctx, QM_ERR_CUDA, "group table overflow in a streamed batch (device status %d)", st.error);
  }
  gt.groups_upper += (int64_t)st.groups_inserted;
  gt.selected += st.rows_selected;
  gt.rows_done += n_rows;
  return QM_OK;
}

}  // namespace

extern "C" {

int qm_agg_begin(qm_ctx *ctx, const qm_query *q, qm_agg **out) {
  if (!ctx || !q || !out) return set_err(ctx, QM_ERR_INVALID, "qm_agg_begin: bad arguments");
  *out = nullptr;
  if (q->flags & QM_FLAG_DETERMINISTIC)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "deterministic float SUM runs through qm_query_run, batches and servers");
  qm_agg *a = new qm_agg();
  a->ctx = ctx;
  // deep copy (names live in a->strs; reserve so c_str() stays valid)
  int n_or = 0;
  for (int g = 0; g < q->n_or_groups; g++) n_or += q->or_group_sizes[g];
  a->strs.reserve(3 + q->n_filters + n_or + q->n_group_by + 2 * q->n_aggregates);
  auto dup = [&](const char *s) -> const char * {
    if (!s) return nullptr;
    a->strs.emplace_back(s);
    return a->strs.back().c_str();
  };
  for (int i = 0; i < q->n_filters; i++) {
    qm_filter f = q->filters[i];
    f.column = dup(f.column);
    a->filters.push_back(f);
  }
  for (int i = 0; i < n_or; i++) {
    qm_filter f = q->or_filters[i];
    f.column = dup(f.column);
    a->or_filters.push_back(f);
  }
  for (int g = 0; g < q->n_or_groups; g++) a->or_sizes.push_back(q->or_group_sizes[g]);
  for (int i = 0; i < q->n_group_by; i++) a->group_by.push_back(dup(q->group_by[i]));
  for (int i = 0; i < q->n_aggregates; i++) {
    qm_aggregate ag = q->aggregates[i];
    ag.column = dup(ag.column);
    ag.alias = dup(ag.alias);
    a->aggs.push_back(ag);
  }
  a->q = *q;
  a->q.order_by = dup(q->order_by);
  a->q.filters = a->filters.data();
  a->q.or_filters = a->or_filters.data();
  a->q.or_group_sizes = a->or_sizes.data();
  a->q.group_by = a->group_by.data();
  a->q.aggregates = a->aggs.data();
  *out = a;
  return QM_OK;
}

int qm_agg_push(qm_agg *a, int64_t n_rows, int32_t n_cols, const qm_column *cols, const uint32_t *selection,
                int64_t n_selected) {
  if (!a) return QM_ERR_INVALID;
  qm_ctx *ctx = a->ctx;
  if (a->failed) return set_err(ctx, QM_ERR_INVALID, "aggregation already failed");
  if (n_rows < 0 || n_cols < 0 || (n_cols > 0 && !cols) || (selection && n_selected < 0))
    return set_err(ctx, QM_ERR_INVALID, "qm_agg_push: bad arguments");
  if (n_rows > 0xffffffffLL) return set_err(ctx, QM_ERR_UNSUPPORTED, "batches are limited to 2^32-1 rows");
  cudaSetDevice(ctx->device);
  // schema is fixed by the first push
  if (!a->planned) {
    for (int i = 0; i < n_cols; i++) a->schema.push_back({cols[i].name ? cols[i].name : "", cols[i].dtype});
  } else {
    for (int i = 0; i < n_cols; i++) {
      bool ok = false;
      for (auto &sc : a->schema)
        if (cols[i].name && sc.first == cols[i].name) ok = sc.second == cols[i].dtype;
      if (!ok) return set_err(ctx, QM_ERR_INVALID, "column %s changed type or was not in the first batch",
                              cols[i].name ? cols[i].name : "?");
    }
  }
  std::vector<DevCol> dcols;
  int rc = stage_batch(ctx, n_rows, n_cols, cols, dcols);
  if (rc) return rc;
  const uint32_t *dsel = nullptr;
  if ((rc = stage_selection(ctx, selection, n_selected, &dsel))) return rc;
  if (dsel && n_selected > 0) {
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
    CK(qm_launch_check_selection(dsel, n_selected, n_rows, (qm_status *)ctx->status.p, ctx->sm_count, ctx->stream));
    qm_status cst;
    if ((rc = read_status(ctx, &cst))) return rc;
    if (cst.error) return set_err(ctx, QM_ERR_INVALID, "selection is not strictly ascending row indices below %lld",
                                  (long long)n_rows);
  }
  const int64_t n_elems = selection ? n_selected : n_rows;
  ColEnv env;
  for (auto &c : dcols) env.views.push_back({&c, n_rows});
  return agg_push_env(a, env, n_rows, dsel, n_elems);
}

int qm_agg_push_table(qm_agg *a, const qm_table *table) {
  if (!a || !table) return QM_ERR_INVALID;
  qm_ctx *ctx = a->ctx;
  if (a->failed) return set_err(ctx, QM_ERR_INVALID, "aggregation already failed");
  if (table->ctx != ctx) return set_err(ctx, QM_ERR_INVALID, "table of another context");
  if (table->n_rows > 0xffffffffLL) return set_err(ctx, QM_ERR_UNSUPPORTED, "batches are limited to 2^32-1 rows");
  cudaSetDevice(ctx->device);
  if (!a->planned)
    for (auto &c : table->cols) a->schema.push_back({c.name, c.dtype});
  ColEnv env;
  for (auto &c : table->cols) env.views.push_back({&c, table->n_rows});
  return agg_push_env(a, env, table->n_rows, nullptr, table->n_rows);
}

int qm_agg_finish(qm_agg *a, qm_result **out) {
  if (!a || !out) return QM_ERR_INVALID;
  qm_ctx *ctx = a->ctx;
  *out = nullptr;
  if (a->failed) return set_err(ctx, QM_ERR_INVALID, "aggregation failed earlier");
  cudaSetDevice(ctx->device);
  if (!a->planned) {
    // no batch at all: plan against an empty schema is impossible when the
    // query names columns; an ungrouped COUNT(*) still has its one row
    std::vector<DevCol> none;
    ColEnv env;
    GroupTable &gt = a->gt;
    int rc = plan_query(ctx, &a->q, env, gt.pl);
    if (rc) return rc;
    gt.pl.key.mode = gt.pl.key.n_cols == 0 ? QK_NONE : QK_HASH;
    if ((rc = setup_table(ctx, gt, 1, 0, true))) return rc;
    a->planned = true;
  }
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  int rc = finish_table(ctx, a->gt, out, 0.f);
  if (rc) return rc;
  (*out)->stats.rows_scanned = a->gt.rows_done;
  (*out)->stats.bytes_scanned = a->gt.pl.bytes_per_row * a->gt.rows_done;
  (*out)->stats.device_ms += a->device_ms;
  return QM_OK;
}

int qm_agg_destroy(qm_agg *a) {
  if (!a) return QM_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  // keep the larger of this table and the spare for the next aggregation
  if (a->gt.own.bytes > a->ctx->agg_spare.bytes) std::swap(a->gt.own, a->ctx->agg_spare);
  release(a->gt.own);
  delete a;
  return QM_OK;
}

int qm_agg_partial_export(qm_agg *a, int64_t row_offset, uint64_t *dst, int64_t capacity_rows, int64_t *n_groups,
                          int32_t *row_words) {
  if (!a || !n_groups || !row_words || row_offset < 0 || (dst && capacity_rows < 0)) return QM_ERR_INVALID;
  qm_ctx *ctx = a->ctx;
  if (a->failed) return set_err(ctx, QM_ERR_INVALID, "aggregation failed earlier");
  if (!a->planned) return set_err(ctx, QM_ERR_INVALID, "partial export before the first push");
  cudaSetDevice(ctx->device);
  GroupTable &gt = a->gt;
  const Exec &ex = gt.ex;
  *row_words = ex.stride + 1;
  int64_t G = 1;
  const uint32_t *slots = nullptr;
  if (gt.pl.key.mode != QK_NONE) {
    int rc;
    if ((rc = ensure(ctx, ctx->keys, ex.total_slots * 8)) || (rc = ensure(ctx, ctx->slots, ex.total_slots * 4)) ||
        (rc = ensure(ctx, ctx->counter, 64)) || (rc = ensure_host(ctx, ctx->hstatus, 64)))
      return rc;
    CK(cudaMemsetAsync(ctx->counter.p, 0, 8, ctx->stream));
    CK(qm_launch_compact(gt.table, ex.total_slots, ex.stride, gt.pl.agg.acc[gt.pl.agg.acc_count].word, -1,
                         (uint64_t *)ctx->keys.p, (uint32_t *)ctx->slots.p, (unsigned long long *)ctx->counter.p,
                         ctx->sm_count, ctx->stream));
    CK(cudaMemcpyAsync(ctx->hstatus.p, ctx->counter.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    G = (int64_t)*(unsigned long long *)ctx->hstatus.p;
    slots = (const uint32_t *)ctx->slots.p;
  }
  *n_groups = G;
  if (!dst) return QM_OK;
  if (G > capacity_rows) return set_err(ctx, QM_ERR_CAPACITY, "partial has %lld groups, room for %lld", (long long)G,
                                        (long long)capacity_rows);
  CK(qm_launch_export_partial(gt.table, ex.stride, slots, G, ex.n_slots, gt.pl.key.mode, gt.pl.agg, row_offset, dst,
                              ctx->sm_count, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return QM_OK;
}

int qm_agg_partial_merge(qm_agg *a, const uint64_t *src, int64_t n_groups, int32_t row_words, int64_t rows_end) {
  if (!a || (n_groups > 0 && !src) || n_groups < 0 || rows_end < 0) return QM_ERR_INVALID;
  qm_ctx *ctx = a->ctx;
  if (a->failed) return set_err(ctx, QM_ERR_INVALID, "aggregation failed earlier");
  if (!a->planned) return set_err(ctx, QM_ERR_INVALID, "partial merge before the first push");
  GroupTable &gt = a->gt;
  if (row_words != gt.ex.stride + 1)
    return set_err(ctx, QM_ERR_INVALID, "partial rows of %d words; this aggregation's are %d", row_words,
                   gt.ex.stride + 1);
  cudaSetDevice(ctx->device);
  int rc;
  if (gt.pl.key.mode == QK_HASH && (rc = grow_table(ctx, gt, gt.groups_upper + n_groups))) return rc;
  qm_scan_args args;
  fill_args(gt, args, (qm_status *)ctx->status.p);
  CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
  CK(qm_launch_merge_partial(args, src, n_groups, ctx->sm_count, ctx->stream));
  qm_status st;
  if ((rc = read_status(ctx, &st))) return rc;
  if (st.error) {
    a->failed = true;
    return set_err(ctx, QM_ERR_CUDA, "group table overflow while merging a partial (device status %d)", st.error);
  }
  gt.groups_upper += (int64_t)st.groups_inserted;
  gt.rows_done = std::max(gt.rows_done, rows_end);
  return QM_OK;
}

int qm_agg_partial_layout(const qm_agg *a, int32_t *row_words, int32_t *first_word) {
  if (!a || !row_words || !first_word) return QM_ERR_INVALID;
  if (!a->planned) return set_err(a->ctx, QM_ERR_INVALID, "partial layout before the first push");
  *row_words = a->gt.ex.stride + 1;
  *first_word = a->gt.pl.agg.w_first >= 0 ? 2 + a->gt.pl.agg.w_first : -1;
  return QM_OK;
}

int qm_agg_partial_begin(const qm_agg *src, qm_agg **out) {
  if (!src || !out) return QM_ERR_INVALID;
  *out = nullptr;
  qm_ctx *ctx = src->ctx;
  if (!src->planned) return set_err(ctx, QM_ERR_INVALID, "partial begin from an aggregation without a push");
  cudaSetDevice(ctx->device);
  qm_agg *a = nullptr;
  int rc = qm_agg_begin(ctx, &src->q, &a);
  if (rc) return rc;
  a->gt.pl = src->gt.pl;
  a->schema = src->schema;
  if ((rc = setup_table(ctx, a->gt, 1, 0, true))) {
    qm_agg_destroy(a);
    return rc;
  }
  a->planned = true;
  *out = a;
  return QM_OK;
}

int qm_partial_partition(qm_ctx *ctx, const uint64_t *src, int64_t n_rows, int32_t row_words, int32_t parts,
                         uint64_t *dst, int64_t *part_rows) {
  if (!ctx || n_rows < 0 || (n_rows > 0 && (!src || !dst)) || row_words < 2 || parts < 1 || parts > 4096 ||
      !part_rows)
    return set_err(ctx, QM_ERR_INVALID, "qm_partial_partition: bad arguments");
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = ensure(ctx, ctx->counts, sizeof(unsigned long long) * 2 * parts)) ||
      (rc = ensure_host(ctx, ctx->hout, sizeof(unsigned long long) * parts)))
    return rc;
  unsigned long long *cnt = (unsigned long long *)ctx->counts.p, *cur = cnt + parts;
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * parts, ctx->stream));
  CK(qm_launch_partition_count(src, n_rows, row_words, parts, cnt, ctx->sm_count, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hout.p, cnt, sizeof(unsigned long long) * parts, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<unsigned long long> start(parts);
  unsigned long long acc = 0;
  for (int p = 0; p < parts; p++) {
    start[p] = acc;
    part_rows[p] = (int64_t)((unsigned long long *)ctx->hout.p)[p];
    acc += (unsigned long long)part_rows[p];
  }
  CK(cudaMemcpyAsync(cur, start.data(), sizeof(unsigned long long) * parts, cudaMemcpyHostToDevice, ctx->stream));
  CK(qm_launch_partition_scatter(src, n_rows, row_words, parts, cur, dst, ctx->sm_count, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return QM_OK;
}

int qm_filter_select(qm_ctx *ctx, int64_t n_rows, int32_t n_cols, const qm_column *cols, const qm_query *q,
                     const uint32_t *selection, int64_t n_selected, uint32_t *out_indices, int64_t max_out,
                     int64_t *out_count) {
  if (!ctx || !q || !out_count || n_rows < 0 || (n_cols > 0 && !cols) || max_out < 0 || (max_out > 0 && !out_indices) ||
      (selection && n_selected < 0))
    return set_err(ctx, QM_ERR_INVALID, "qm_filter_select: bad arguments");
  if (n_rows > 0xffffffffLL) return set_err(ctx, QM_ERR_UNSUPPORTED, "batches are limited to 2^32-1 rows");
  cudaSetDevice(ctx->device);
  *out_count = 0;
  std::vector<DevCol> dcols;
  int rc = stage_batch(ctx, n_rows, n_cols, cols, dcols);
  if (rc) return rc;
  ColEnv env;
  for (auto &c : dcols) env.views.push_back({&c, n_rows});
  qm_pred P;
  std::vector<const DevCol *> touched;
  int64_t bpr = 0;
  if ((rc = build_pred(ctx, q, env, P, bpr, touched))) return rc;
  const uint32_t *dsel = nullptr;
  if ((rc = stage_selection(ctx, selection, n_selected, &dsel))) return rc;
  if (dsel && n_selected > 0) {
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(qm_status), ctx->stream));
    CK(qm_launch_check_selection(dsel, n_selected, n_rows, (qm_status *)ctx->status.p, ctx->sm_count, ctx->stream));
    qm_status cst;
    if ((rc = read_status(ctx, &cst))) return rc;
    if (cst.error) return set_err(ctx, QM_ERR_INVALID, "selection is not strictly ascending row indices below %lld",
                                  (long long)n_rows);
  }
  const int64_t n_elems = selection ? n_selected : n_rows;
  if (n_elems == 0) return QM_OK;
  const int64_t n_tiles = (n_elems + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
  if ((rc = ensure(ctx, ctx->masks, (size_t)n_tiles * QM_R * 4)) || (rc = ensure(ctx, ctx->counts, (size_t)n_tiles * 4 + 4)) ||
      (rc = ensure(ctx, ctx->offsets, (size_t)(n_tiles + 1) * 8)) || (rc = ensure_host(ctx, ctx->hstatus, 64)))
    return rc;
  CK(qm_launch_select_masks(P, n_elems, dsel, (uint32_t *)ctx->masks.p, (uint32_t *)ctx->counts.p, ctx->sm_count,
                            ctx->stream));
  size_t tb = 0;
  CK(qm_exclusive_scan_u32(nullptr, &tb, (uint32_t *)ctx->counts.p, (uint64_t *)ctx->offsets.p, n_tiles + 1,
                           ctx->stream));
  if ((rc = ensure(ctx, ctx->sort_temp, tb))) return rc;
  tb = ctx->sort_temp.bytes;
  // counts[n_tiles] = 0 so offsets[n_tiles] is the total
  CK(cudaMemsetAsync((uint32_t *)ctx->counts.p + n_tiles, 0, 4, ctx->stream));
  CK(qm_exclusive_scan_u32(ctx->sort_temp.p, &tb, (uint32_t *)ctx->counts.p, (uint64_t *)ctx->offsets.p,
                           n_tiles + 1, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hstatus.p, (uint64_t *)ctx->offsets.p + n_tiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t total = (int64_t)*(uint64_t *)ctx->hstatus.p;
  *out_count = total;
  const int64_t n_write = std::min(total, max_out);
  if (n_write > 0) {
    if ((rc = ensure(ctx, ctx->sel_out, (size_t)n_write * 4 + 16))) return rc;
    CK(qm_launch_select_write(n_tiles, dsel, (uint32_t *)ctx->masks.p, (uint64_t *)ctx->offsets.p,
                              (uint32_t *)ctx->sel_out.p, n_write, ctx->sm_count, ctx->stream));
    CK(cudaMemcpyAsync(out_indices, ctx->sel_out.p, (size_t)n_write * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if (total > max_out) return set_err(ctx, QM_ERR_CAPACITY, "%lld rows pass, capacity %lld", (long long)total, (long long)max_out);
  return QM_OK;
}

int qm_result_num_rows(const qm_result *r, int64_t *out) {
  if (!r || !out) return QM_ERR_INVALID;
  *out = r->n_rows;
  return QM_OK;
}

int qm_result_num_columns(const qm_result *r, int32_t *out) {
  if (!r || !out) return QM_ERR_INVALID;
  *out = (int32_t)r->cols.size();
  return QM_OK;
}

int qm_result_column(const qm_result *r, int32_t i, qm_result_col *out) {
  if (!r || !out || i < 0 || i >= (int32_t)r->cols.size()) return QM_ERR_INVALID;
  const auto &c = r->cols[i];
  out->name = c.name.c_str();
  out->dtype = c.dtype;
  out->is_key = c.is_key;
  out->n_rows = r->n_rows;
  out->data = c.data;
  out->null_bitmap = c.has_nulls ? c.nulls : nullptr;
  return QM_OK;
}

int qm_result_stats(const qm_result *r, qm_stats *out) {
  if (!r || !out) return QM_ERR_INVALID;
  *out = r->stats;
  return QM_OK;
}

int qm_result_qmcb(const qm_result *cr, const uint8_t **buf, size_t *len) {
  if (!cr || !buf || !len) return QM_ERR_INVALID;
  qm_result *r = const_cast<qm_result *>(cr);
  if (!r->qmcb_built) {
    // encodeColumnarBatch layout (src/columnar.ts:523-613)
    std::vector<uint8_t> &o = r->qmcb;
    o.clear();
    auto put = [&](const void *p, size_t n) { o.insert(o.end(), (const uint8_t *)p, (const uint8_t *)p + n); };
    uint32_t magic = 0x42434D51u, rows = (uint32_t)r->n_rows;
    uint16_t nc = (uint16_t)r->cols.size();
    put(&magic, 4);
    put(&rows, 4);
    put(&nc, 2);
    std::vector<int> tags;
    for (auto &c : r->cols) {
      int tag = c.dtype;
      if (c.dtype == QM_I128) {
        for (int64_t i = 0; i < r->n_rows; i++) {
          uint64_t lo;
          int64_t hi;
          memcpy(&lo, c.data + 16 * i, 8);
          memcpy(&hi, c.data + 16 * i + 8, 8);
          if (hi != ((int64_t)lo < 0 ? -1 : 0)) return QM_ERR_UNSUPPORTED;
        }
        tag = QM_I64;
      }
      tags.push_back(tag);
      uint16_t nl = (uint16_t)c.name.size();
      put(&nl, 2);
      put(c.name.data(), nl);
      uint8_t t8 = (uint8_t)tag, hn = c.has_nulls ? 1 : 0;
      put(&t8, 1);
      put(&hn, 1);
    }
    for (size_t k = 0; k < r->cols.size(); k++) {
      auto &c = r->cols[k];
      if (c.has_nulls) put(c.nulls, (size_t)((r->n_rows + 7) / 8));
      if (c.dtype == QM_I128) {
        for (int64_t i = 0; i < r->n_rows; i++) put(c.data + 16 * i, 8);
      } else {
        put(c.data, c.bytes);
      }
    }
    r->qmcb_built = true;
  }
  *buf = r->qmcb.data();
  *len = r->qmcb.size();
  return QM_OK;
}

int qm_result_destroy(qm_result *r) {
  delete r;
  return QM_OK;
}

}  // extern "C"

// ================================================================ no-alloc
// qm_query_run_noalloc: the filter -> GROUP BY of qm_query_run for callers
// that cannot allocate device memory — code running inside another
// framework's memory manager or arena, or while the device allocator is
// unavailable to it.  Every temporary (group table, device status word,
// compaction lists, staged result columns) lives in one file-scope static
// device array of QM_NOALLOC_SCRATCH_BYTES that each device holds from the
// library's first use until the process exits.  The host code of this file
// reaches it through cudaGetSymbolAddress, once per device (the array's
// name is only a host-side stand-in).  Calls share the array: overlapping
// calls on the GPU race and must be serialised by the caller.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QM_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_addr[128];
bool g_noalloc_ready[128];

// The device address of the scratch array on the current device (set up on
// the first call per device; that call must come before any stream capture).
// The address is kept for the life of the process: it does not survive a
// cudaDeviceReset (or a primary context torn down and created again), after
// which this entry point must not be called on that device.
int noalloc_scratch(qm_ctx *ctx, unsigned char **out) {
  if (ctx->device < 0 || ctx->device >= 128) return set_err(ctx, QM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ready[ctx->device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_err(ctx, QM_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    }
    g_noalloc_addr[ctx->device] = p;
    g_noalloc_ready[ctx->device] = true;
  }
  *out = (unsigned char *)g_noalloc_addr[ctx->device];
  return QM_OK;
}

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int qm_query_run_noalloc(qm_ctx *ctx, int64_t n_rows, int32_t n_cols, const qm_column *cols,
                                    const qm_query *q, int64_t max_groups, void *const *out_columns,
                                    uint32_t *const *out_null_words, int32_t *out_dtypes, int64_t *out_groups) {
  if (!ctx || !q || !out_columns || !out_groups || n_rows < 0 || n_cols < 0 || (n_cols > 0 && !cols) ||
      max_groups <= 0)
    return set_err(ctx, QM_ERR_INVALID, "qm_query_run_noalloc: bad arguments");
  if (n_rows > 0xffffffffLL) return set_err(ctx, QM_ERR_UNSUPPORTED, "batches are limited to 2^32-1 rows");
  if (q->order_by || q->has_limit || q->offset)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "ORDER BY / LIMIT / OFFSET run through qm_query_run");
  if (q->flags & QM_FLAG_DETERMINISTIC)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "deterministic float SUM needs column statistics: qm_query_run");
  *out_groups = 0;
  // no group needs less than 8 bytes of scratch: a larger capacity cannot
  // fit, and bounding it here keeps the size arithmetic below from overflowing
  if (max_groups > (int64_t)(QM_NOALLOC_SCRATCH_BYTES / 8))
    return set_err(ctx, QM_ERR_CAPACITY, "max_groups = %lld cannot fit the %u-byte scratch array",
                   (long long)max_groups, (unsigned)QM_NOALLOC_SCRATCH_BYTES);
  cudaSetDevice(ctx->device);
  unsigned char *scratch = nullptr;
  int rc = noalloc_scratch(ctx, &scratch);
  if (rc) return rc;
  // columns are read in place: device memory only, NULL bitmaps readable as
  // ceil(n_rows / 32) 32-bit words
  std::vector<DevCol> dcols(n_cols);
  for (int i = 0; i < n_cols; i++) {
    const qm_column &c = cols[i];
    if (!c.name || !valid_dtype(c.dtype)) return set_err(ctx, QM_ERR_INVALID, "column %d: name / dtype", i);
    if (!c.on_device) return set_err(ctx, QM_ERR_INVALID, "column %s: qm_query_run_noalloc reads device columns only", c.name);
    if (n_rows > 0 && !c.data) return set_err(ctx, QM_ERR_INVALID, "column %s: no data", c.name);
    if (c.null_bitmap && ((uintptr_t)c.null_bitmap & 3))
      return set_err(ctx, QM_ERR_INVALID, "column %s: NULL bitmap must be 4-byte aligned", c.name);
    dcols[i].name = c.name;
    dcols[i].dtype = c.dtype;
    dcols[i].data = const_cast<void *>(c.data);
    dcols[i].nulls = (uint32_t *)c.null_bitmap;
  }
  ColEnv env;
  for (auto &c : dcols) env.views.push_back({&c, n_rows});
  GroupTable gt;
  if ((rc = plan_query(ctx, q, env, gt.pl))) return rc;
  Plan &pl = gt.pl;
  uint64_t space = 0;
  if ((rc = plan_key_packing(ctx, pl, n_rows, false, &space))) return rc;
  pl.key.mode = pl.key.n_cols == 0 ? QK_NONE : QK_HASH;
  if (out_dtypes)
    for (int k = 0; k < pl.outs.n_out; k++) out_dtypes[k] = pl.outs.o[k].dtype;
  for (int k = 0; k < pl.outs.n_out; k++)
    if (!out_columns[k]) return set_err(ctx, QM_ERR_INVALID, "output column %d has no buffer", k);
  // sizes inside the scratch array
  Exec &ex = gt.ex;
  if (pl.key.mode == QK_NONE) {
    ex.n_slots = 1;
  } else {
    ex.log2cap = ilog2_ceil(std::max<int64_t>(1024, max_groups * 2 + max_groups / 8));
    if (ex.log2cap > 30) return set_err(ctx, QM_ERR_CAPACITY, "max_groups too large for the scratch array");
    ex.n_slots = (int64_t)1 << ex.log2cap;
  }
  choose_layout(pl, max_groups, ex, ctx->tuning);
  const int64_t G_cap = pl.key.mode == QK_NONE ? 1 : max_groups;
  const size_t status_off = 0;
  const size_t table_off = 256;
  const size_t table_bytes = up256((size_t)ex.total_slots * ex.stride * 8);
  const size_t keys_off = table_off + table_bytes;
  const size_t slots_off = keys_off + up256((size_t)ex.total_slots * 8);
  const size_t out_off = slots_off + up256((size_t)ex.total_slots * 4);
  qm_outspec O = pl.outs;
  size_t off = 0;
  const size_t null_words_bytes = (size_t)((G_cap + 31) / 32) * 4;
  for (int k = 0; k < O.n_out; k++) {
    O.o[k].offset = (int64_t)off;
    off += up256((size_t)G_cap * dtype_size(O.o[k].dtype));
    if (pl.meta[k].nullable) {
      O.o[k].null_offset = (int64_t)off;
      off += up256(null_words_bytes);
    } else {
      O.o[k].null_offset = -1;
    }
  }
  const size_t need = out_off + off;
  if (need > (size_t)QM_NOALLOC_SCRATCH_BYTES)
    return set_err(ctx, QM_ERR_CAPACITY,
                   "query needs %zu bytes of scratch for %lld groups; the fixed scratch array holds %u bytes",
                   need, (long long)max_groups, (unsigned)QM_NOALLOC_SCRATCH_BYTES);
  qm_status *status = (qm_status *)(scratch + status_off);
  gt.table = (uint64_t *)(scratch + table_off);
  // status starts at zero; the group table is re-initialised every call
  CK(cudaMemsetAsync(status, 0, sizeof(qm_status), ctx->stream));
  if ((rc = init_table(ctx, gt))) return rc;
  if (n_rows > 0) {
    qm_scan_args a;
    fill_args(gt, a, status);
    a.n = n_rows;
    a.sel = nullptr;
    a.row_offset = 0;
    // per-warp copies pay only on large inputs (the rule of run_scan)
    if (a.priv && n_rows < PRIV_MIN_ROWS) a.priv = 0;
    const size_t smem = qm_scan_smem_bytes(ex.local_slots, ex.local_hash, pl.agg.n_words, 0, 0, a.priv);
    const int blocks = scan_blocks(ctx, smem, n_rows, false);
    CK(qm_launch_scan(a, blocks, smem, ctx->stream));
  }
  qm_status st;
  CK(cudaMemcpyAsync(&st, status, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (st.error == QM_DEV_OVERFLOW)
    return set_err(ctx, QM_ERR_CAPACITY, "more groups than max_groups = %lld", (long long)max_groups);
  if (st.error) return set_err(ctx, QM_ERR_CUDA, "device status %d", st.error);
  int64_t G = 1;
  const uint32_t *slots = nullptr;
  if (pl.key.mode != QK_NONE) {
    unsigned long long *counter = (unsigned long long *)((unsigned char *)status + offsetof(qm_status, groups_inserted));
    CK(cudaMemsetAsync(counter, 0, 8, ctx->stream));
    CK(qm_launch_compact(gt.table, ex.total_slots, ex.stride, pl.agg.w_count, -1, (uint64_t *)(scratch + keys_off),
                         (uint32_t *)(scratch + slots_off), counter, ctx->sm_count, ctx->stream));
    unsigned long long g = 0;
    CK(cudaMemcpyAsync(&g, counter, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    G = (int64_t)g;
    if (G > max_groups) return set_err(ctx, QM_ERR_CAPACITY, "%lld groups exceed max_groups = %lld", (long long)G,
                                       (long long)max_groups);
    slots = (const uint32_t *)(scratch + slots_off);
  }
  unsigned char *outbase = scratch + out_off;
  CK(cudaMemsetAsync(outbase, 0, off, ctx->stream));
  CK(qm_launch_emit(gt.table, ex.stride, slots, G, pl.key, ex.n_slots, O, outbase, ctx->sm_count, ctx->stream));
  for (int k = 0; k < O.n_out; k++) {
    if (G > 0)
      CK(cudaMemcpyAsync(out_columns[k], outbase + O.o[k].offset, (size_t)G * dtype_size(O.o[k].dtype),
                         cudaMemcpyDeviceToDevice, ctx->stream));
    if (out_null_words && out_null_words[k]) {
      const size_t nw = (size_t)((G + 31) / 32) * 4;
      if (O.o[k].null_offset >= 0) {
        if (nw) CK(cudaMemcpyAsync(out_null_words[k], outbase + O.o[k].null_offset, nw, cudaMemcpyDeviceToDevice, ctx->stream));
      } else if (nw) {
        CK(cudaMemsetAsync(out_null_words[k], 0, nw, ctx->stream));
      }
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  *out_groups = G;
  return QM_OK;
}

// ================================================================== batches
// Many queries, each over its own registered table, in one persistent fused
// launch (qm_batch.cu) captured as a CUDA graph on the first run and
// replayed afterwards.  The work split (tiles per chunk), the block-local
// table budget and blocks per SM are the autotuner's knobs.
#include "qm_batch.h"

namespace {

// Keeps a batch run's packed pinned buffer alive for all of its results.
struct SharedPinned {
  std::shared_ptr<PinnedPool> pool;
  HostBuf buf;
  ~SharedPinned() {
    if (pool) pool->release(buf);
  }
};

int64_t region_bytes(int64_t G, const qm_bq &b) {
  int64_t off = 0;
  for (int k = 0; k < b.outs.n_out; k++) {
    off += (G * b.width[k] + 15) & ~(int64_t)15;
    if (b.nullable[k]) off += ((G + 31) / 32 * 4 + 15) & ~(int64_t)15;
  }
  return off;
}

// A deep copy of a qm_query (the caller's strings and arrays may go away
// once submit returns).
struct OwnedQuery {  // holds pointers into itself: never copied or moved
  OwnedQuery() = default;
  OwnedQuery(const OwnedQuery &) = delete;
  OwnedQuery &operator=(const OwnedQuery &) = delete;
  std::deque<std::string> strs;  // deque: stable addresses
  std::vector<qm_filter> filters, or_filters;
  std::vector<int32_t> or_sizes;
  std::vector<const char *> group_by;
  std::vector<qm_aggregate> aggs;
  qm_query q{};

  const char *keep(const char *p) {
    if (!p) return nullptr;
    strs.emplace_back(p);
    return strs.back().c_str();
  }
  void copy(const qm_query &src) {
    q = src;
    for (int i = 0; i < src.n_filters; i++) {
      qm_filter f = src.filters[i];
      f.column = keep(f.column);
      filters.push_back(f);
    }
    int64_t n_or = 0;
    for (int g = 0; g < src.n_or_groups; g++) {
      or_sizes.push_back(src.or_group_sizes[g]);
      n_or += src.or_group_sizes[g];
    }
    for (int64_t i = 0; i < n_or; i++) {
      qm_filter f = src.or_filters[i];
      f.column = keep(f.column);
      or_filters.push_back(f);
    }
    for (int i = 0; i < src.n_group_by; i++) group_by.push_back(keep(src.group_by[i]));
    for (int i = 0; i < src.n_aggregates; i++) {
      qm_aggregate a = src.aggregates[i];
      a.column = keep(a.column);
      a.alias = keep(a.alias);
      aggs.push_back(a);
    }
    q.filters = filters.empty() ? nullptr : filters.data();
    q.or_group_sizes = or_sizes.empty() ? nullptr : or_sizes.data();
    q.or_filters = or_filters.empty() ? nullptr : or_filters.data();
    q.group_by = group_by.empty() ? nullptr : group_by.data();
    q.aggregates = aggs.empty() ? nullptr : aggs.data();
    q.order_by = keep(src.order_by);
  }
};

}  // namespace

// One wave of a batched run: a contiguous slice [q0, q1) of the batch's
// queries in wave order, with its own finalize buffers, so that its packed
// results cross the host link while later waves scan.
struct BatchWave {
  int q0 = 0, q1 = 0;     // positions in the batch's wave order
  int64_t slots = 0;      // group-table slots of its queries
  int64_t bm_words = 0;   // words of its first-row bitmap
  qm_batch_dev dev{};
  // mode 0: one persistent launch per query class present in the wave, over
  // chunks [chunk0, chunk0 + n_chunks) of the wave's chunk list
  struct ClassLaunch {
    int cls, chunk0, n_chunks, blocks, local_bytes;
    size_t smem;
  };
  std::vector<ClassLaunch> classes;
  DevBuf d_slot0, d_chunks, d_bitmap, d_popc, d_ranks, d_temp, d_meta, d_packed, d_nullbytes, d_perm;
  HostBuf h_meta;         // pinned: the wave's layout, copied back with its work
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t done = nullptr;  // the wave's device work ended (results packed, layout copied)
  std::shared_ptr<SharedPinned> host;  // its packed results in host memory
  ~BatchWave() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (done) cudaEventDestroy(done);
    DevBuf *bufs[] = {&d_slot0, &d_chunks, &d_bitmap, &d_popc, &d_ranks, &d_temp, &d_meta, &d_packed, &d_nullbytes,
                      &d_perm};
    for (DevBuf *b : bufs) release(*b);
    if (h_meta.p) cudaFreeHost(h_meta.p);
  }
};

struct qm_batch {
  qm_ctx *ctx = nullptr;
  int n = 0;
  std::vector<GroupTable> gts;  // per query, in the caller's order
  std::vector<qm_bq> bq;
  std::vector<int64_t> rows;
  std::vector<int64_t> est;  // planner's group estimate per query
  std::vector<Exec> ex_plan;  // the planner's block-local layout per query (mode 1)
  struct Launch {
    qm_scan_args a;
    int blocks;
    size_t smem;
  };
  std::vector<Launch> launches;       // mode 1: one specialised scan per query
  std::vector<int> order;             // wave position -> query
  std::vector<int> pos;               // query -> wave position
  std::vector<int> wave_of;           // wave position -> wave
  std::vector<std::unique_ptr<BatchWave>> waves;
  int waves_req = 0;                  // waves asked for (0: by batch size)
  std::vector<cudaStream_t> side;     // mode 1: branches the launches spread over
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  cudaStream_t stream = nullptr;      // the batch's work (null: the context's stream)
  cudaStream_t copy_stream = nullptr; // result copies
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
  std::vector<cudaEvent_t> q_ev;      // per-query copies landed (per-request completion)
  std::vector<std::shared_ptr<SharedPinned>> q_host;  // per-request result buffers until completed
  int mode = 1;  // 0: persistent kernels (one per query class) over (query, chunk) work items; 1: per-query launches
  std::vector<const qm_table *> tabs;  // query i's table and a copy of the
  std::vector<std::unique_ptr<OwnedQuery>> queries;  // query, to rerun it alone
  DevBuf arena, d_bq, d_counter, d_status;
  HostBuf h_status;  // pinned, wave order
  int chunk_tiles = 512;
  int local_kb = 40;
  int bps = 0;
  float last_ms = 0;
  int64_t bytes_scanned = 0;
  int64_t total_rows = 0;
  ~qm_batch() {
    waves.clear();
    for (cudaStream_t st : side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : side_ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : q_ev) cudaEventDestroy(ev);
    if (fork_ev) cudaEventDestroy(fork_ev);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_end) cudaEventDestroy(ev_end);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    DevBuf *bufs[] = {&arena, &d_bq, &d_counter, &d_status};
    for (DevBuf *b : bufs) release(*b);
    if (h_status.p) cudaFreeHost(h_status.p);
  }
  cudaStream_t st() const { return stream ? stream : ctx->stream; }
};

namespace {

void drop_graph(qm_batch *b) {
  for (auto &w : b->waves) {
    if (w->gexec) cudaGraphExecDestroy(w->gexec);
    if (w->graph) cudaGraphDestroy(w->graph);
    w->gexec = nullptr;
    w->graph = nullptr;
  }
}

// Result bytes of query i as planned (its group estimate, capped by rows).
int64_t est_result_bytes(const qm_batch *b, int i) {
  const qm_bq &q = b->bq[i];
  const int64_t G = q.none ? 1 : std::min<int64_t>(std::max<int64_t>(b->est[i], 1), std::max<int64_t>(b->rows[i], 1));
  int64_t w = 0;
  for (int k = 0; k < q.outs.n_out; k++) w += q.width[k];
  return G * w;
}

// Wave order and boundaries: queries whose results are large for the bytes
// they scan first (their copies start early and overlap the rest), queries
// with small results last (the copy after the last wave is short); waves of
// about equal scanned bytes.
void plan_waves(qm_batch *b) {
  const int n = b->n;
  int W = b->waves_req > 0 ? b->waves_req : std::max(1, std::min(8, n / 16));
  W = std::max(1, std::min(W, n));
  b->order.resize(n);
  for (int i = 0; i < n; i++) b->order[i] = i;
  std::vector<double> ratio(n);
  std::vector<int64_t> sb(n);
  int64_t total = 0;
  for (int i = 0; i < n; i++) {
    sb[i] = std::max<int64_t>(b->gts[i].pl.bytes_per_row * b->rows[i], 1) + 4096;
    ratio[i] = (double)est_result_bytes(b, i) / (double)sb[i];
    total += sb[i];
  }
  if (W > 1)
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return ratio[x] > ratio[y]; });
  std::vector<int> cut;  // first wave position of each wave
  cut.push_back(0);
  int64_t acc = 0;
  for (int j = 0; j < n; j++) {
    acc += sb[b->order[j]];
    const int w = (int)cut.size();
    if (w < W && j + 1 < n && (double)acc >= (double)total * w / W) cut.push_back(j + 1);
  }
  cut.push_back(n);
  const int nw = (int)cut.size() - 1;
  while ((int)b->waves.size() > nw) b->waves.pop_back();
  while ((int)b->waves.size() < nw) b->waves.emplace_back(new BatchWave());
  b->pos.assign(n, 0);
  b->wave_of.assign(n, 0);
  for (int w = 0; w < nw; w++) {
    BatchWave &wv = *b->waves[w];
    wv.q0 = cut[w];
    wv.q1 = cut[w + 1];
    // largest query first inside a wave (the parallel branches finish together)
    std::stable_sort(b->order.begin() + wv.q0, b->order.begin() + wv.q1,
                     [&](int x, int y) { return b->rows[x] > b->rows[y]; });
    for (int j = wv.q0; j < wv.q1; j++) b->wave_of[j] = w;
  }
  for (int j = 0; j < n; j++) b->pos[b->order[j]] = j;
}

// (Re)build waves, chunks, table layout and device descriptors for the
// current knobs.
int batch_layout(qm_batch *b) {
  qm_ctx *ctx = b->ctx;
  const int n = b->n;
  cudaStream_t st = b->st();
  const size_t local_budget = (size_t)b->local_kb * 1024;
  int64_t words = 0;
  std::vector<int64_t> table_off(n);
  for (int i = 0; i < n; i++) {
    GroupTable &gt = b->gts[i];
    Exec &ex = gt.ex;
    // block-local table within the batch's shared-memory budget (mode 0)
    const int64_t per_slot = (int64_t)gt.pl.agg.n_words * 8;
    if (ex.local_slots > 0) {
      int64_t need = (int64_t)ex.local_slots * (per_slot + (ex.local_hash ? 8 : 0));
      if (local_budget == 0) {
        ex.local_slots = 0;
      } else if (need > (int64_t)local_budget) {
        int L = 1;
        while ((int64_t)(L * 2) * (per_slot + 8) <= (int64_t)local_budget) L *= 2;
        ex.local_slots = L >= 32 ? L : 0;
        ex.local_hash = 1;
      }
    }
    table_off[i] = words;
    words += ex.total_slots * ex.stride;
  }
  plan_waves(b);
  int rc;
  if ((rc = ensure_on(ctx, b->arena, (size_t)words * 8 + 64, st))) return rc;
  if ((rc = ensure_on(ctx, b->d_status, sizeof(qm_status) * n, st))) return rc;
  if ((rc = ensure_on(ctx, b->d_bq, sizeof(qm_bq) * n, st))) return rc;
  if ((rc = ensure_on(ctx, b->d_counter, sizeof(int) * QM_BATCH_CLASS_SLOTS * b->waves.size(), st))) return rc;
  // sized for the largest batch once: regrowing pinned memory frees the old
  // buffer, which synchronises the device under other batches in flight
  if ((rc = ensure_host(ctx, b->h_status, sizeof(qm_status) * QM_BATCH_MAX))) return rc;
  std::vector<qm_bq> dbq(n);
  for (int i = 0; i < n; i++) {
    GroupTable &gt = b->gts[i];
    gt.table = (uint64_t *)b->arena.p + table_off[i];
    qm_bq &q = b->bq[i];
    fill_args(gt, q.a, (qm_status *)b->d_status.p + b->pos[i]);
    q.a.priv = 0;  // the persistent kernels keep one block-local copy
    q.a.n = b->rows[i];
    q.a.sel = nullptr;
    q.a.row_offset = 0;
    memset(&q.a.stage, 0, sizeof q.a.stage);
  }
  // per query class (dedupe flag, value columns, key kind): the largest local
  // table of its queries sets that persistent kernel's shared memory
  std::vector<int> cls(n);
  int class_local[QM_BATCH_CLASSES_N] = {0};
  for (int i = 0; i < n; i++) {
    const Exec &ex = b->gts[i].ex;
    cls[i] = qm_batch_class_of(b->bq[i].a);
    if (ex.local_slots > 0)
      class_local[cls[i]] = std::max<int>(
          class_local[cls[i]], ex.local_slots * (b->gts[i].pl.agg.n_words * 8 + (ex.local_hash ? 8 : 0)));
  }
  size_t class_smem[QM_BATCH_CLASSES_N];
  int class_bps[QM_BATCH_CLASSES_N];
  for (int c = 0; c < QM_BATCH_CLASSES_N; c++) {
    class_smem[c] = qm_batch_smem_bytes(class_local[c]);
    class_bps[c] = 0;
    bool used = false;
    for (int i = 0; i < n && !used; i++) used = cls[i] == c;
    if (!used) continue;
    int bps = 1;
    {
      std::lock_guard<std::mutex> lk(g_cfg_mu);
      const auto key = std::make_tuple(ctx->device, c, class_smem[c]);
      auto it = g_occ.find(key);
      if (it != g_occ.end()) {
        bps = it->second;
      } else {
        size_t &lim = g_class_attr[std::make_pair(ctx->device, c)];
        const size_t raise = class_smem[c] > lim ? class_smem[c] : 0;
        if (qm_batch_class_configure(c, raise, class_smem[c], &bps) != cudaSuccess) {
          cudaGetLastError();
          return set_err(ctx, QM_ERR_CUDA, "batched kernel: %zu bytes of shared memory rejected", class_smem[c]);
        }
        if (raise) lim = raise;
        g_occ[key] = bps;
      }
    }
    if (bps < 1) bps = 1;
    if (b->bps > 0 && b->bps < bps) bps = b->bps;
    class_bps[c] = bps;
  }
  // per wave: slots, bitmap slices, chunks (grouped by class) and finalize buffers
  for (size_t w = 0; w < b->waves.size(); w++) {
    BatchWave &wv = *b->waves[w];
    std::vector<int64_t> slot0;
    std::vector<qm_chunk> by_class[QM_BATCH_CLASSES_N];
    int64_t slots = 0, bm_words = 0, packed_max = 0, nullbytes_max = 0;
    for (int j = wv.q0; j < wv.q1; j++) {
      const int i = b->order[j];
      const Exec &ex = b->gts[i].ex;
      qm_bq q = b->bq[i];
      slot0.push_back(slots);
      slots += ex.total_slots;
      q.bm_word0 = bm_words;
      q.bm_words = b->rows[i] / 32 + 1;
      bm_words += q.bm_words;
      const int64_t gmax = q.none ? 1 : std::min<int64_t>(ex.total_slots, std::max<int64_t>(b->rows[i], 1));
      packed_max += region_bytes(gmax, q);
      for (int k = 0; k < q.outs.n_out; k++)
        if (q.nullable[k]) nullbytes_max += (gmax + 15) & ~(int64_t)15;
      dbq[j] = q;
      b->bq[i].bm_word0 = q.bm_word0;
      b->bq[i].bm_words = q.bm_words;
      const int64_t tiles = (b->rows[i] + QM_TILE_ROWS - 1) / QM_TILE_ROWS;
      for (int64_t t0 = 0; t0 < tiles; t0 += b->chunk_tiles) {
        qm_chunk c;
        c.q = j - wv.q0;
        c.pad = 0;
        c.tile0 = t0;
        c.tile1 = std::min<int64_t>(tiles, t0 + b->chunk_tiles);
        by_class[cls[i]].push_back(c);
      }
    }
    std::vector<qm_chunk> chunks;
    wv.classes.clear();
    for (int c = 0; c < QM_BATCH_CLASSES_N; c++) {
      if (by_class[c].empty()) continue;
      BatchWave::ClassLaunch L;
      L.cls = c;
      L.chunk0 = (int)chunks.size();
      L.n_chunks = (int)by_class[c].size();
      L.local_bytes = class_local[c];
      L.smem = class_smem[c];
      L.blocks = std::max(1, std::min(ctx->sm_count * class_bps[c], L.n_chunks));
      wv.classes.push_back(L);
      chunks.insert(chunks.end(), by_class[c].begin(), by_class[c].end());
    }
    wv.slots = slots;
    wv.bm_words = bm_words;
    size_t temp = 0;
    CK(qm_batch_scan_temp_bytes(bm_words, &temp));
    if ((rc = ensure_on(ctx, wv.d_slot0, sizeof(int64_t) * slot0.size(), st)) ||
        (rc = ensure_on(ctx, wv.d_chunks, sizeof(qm_chunk) * std::max<size_t>(chunks.size(), 1), st)) ||
        (rc = ensure_on(ctx, wv.d_bitmap, sizeof(uint32_t) * (bm_words + 1), st)) ||
        (rc = ensure_on(ctx, wv.d_popc, sizeof(uint32_t) * (bm_words + 1), st)) ||
        (rc = ensure_on(ctx, wv.d_ranks, sizeof(uint64_t) * (bm_words + 1), st)) ||
        (rc = ensure_on(ctx, wv.d_temp, temp + 16, st)) || (rc = ensure_on(ctx, wv.d_meta, sizeof(qm_batch_meta), st)) ||
        (rc = ensure_on(ctx, wv.d_packed, (size_t)packed_max + 64, st)) ||
        (rc = ensure_on(ctx, wv.d_nullbytes, (size_t)nullbytes_max + 64, st)) ||
        (rc = ensure_on(ctx, wv.d_perm, sizeof(uint32_t) * (size_t)(slots + 1), st)) ||
        (rc = ensure_host(ctx, wv.h_meta, sizeof(qm_batch_meta))))
      return rc;
    CK(cudaMemcpyAsync(wv.d_slot0.p, slot0.data(), sizeof(int64_t) * slot0.size(), cudaMemcpyHostToDevice, st));
    if (!chunks.empty())
      CK(cudaMemcpyAsync(wv.d_chunks.p, chunks.data(), sizeof(qm_chunk) * chunks.size(), cudaMemcpyHostToDevice, st));
    if (!wv.done) CK(cudaEventCreateWithFlags(&wv.done, cudaEventDisableTiming));
    qm_batch_dev &d = wv.dev;
    d.n = wv.q1 - wv.q0;
    d.sm_count = ctx->sm_count;
    d.bq = (qm_bq *)b->d_bq.p + wv.q0;
    d.slot0 = (int64_t *)wv.d_slot0.p;
    d.total_slots = slots;
    d.chunks = (qm_chunk *)wv.d_chunks.p;
    d.n_chunks = (int)chunks.size();
    d.counter = (int *)b->d_counter.p + QM_BATCH_CLASS_SLOTS * w;
    d.statuses = (qm_status *)b->d_status.p + wv.q0;
    d.bitmap = (uint32_t *)wv.d_bitmap.p;
    d.bm_words = bm_words;
    d.popc = (uint32_t *)wv.d_popc.p;
    d.ranks = (uint64_t *)wv.d_ranks.p;
    d.scan_temp = wv.d_temp.p;
    d.scan_temp_bytes = temp;
    d.meta = (qm_batch_meta *)wv.d_meta.p;
    d.meta_host = (qm_batch_meta *)wv.h_meta.p;
    d.meta_bytes = sizeof(qm_batch_meta);
    d.packed = (unsigned char *)wv.d_packed.p;
    d.nullbytes = (unsigned char *)wv.d_nullbytes.p;
    d.perm = (uint32_t *)wv.d_perm.p;
  }
  // (pageable source: the call returns once the bytes are staged, so dbq may go)
  CK(cudaMemcpyAsync(b->d_bq.p, dbq.data(), sizeof(qm_bq) * n, cudaMemcpyHostToDevice, st));
  // mode 1: each query's own specialised scan, with the planner's block-local
  // layout, on one of several stream branches
  b->launches.resize(n);
  for (int i = 0; i < n; i++) {
    GroupTable g;
    g.pl = b->gts[i].pl;
    g.ex = b->ex_plan[i];
    g.table = b->gts[i].table;
    qm_batch::Launch &L = b->launches[i];
    fill_args(g, L.a, (qm_status *)b->d_status.p + b->pos[i]);
    L.a.n = b->rows[i];
    L.a.sel = nullptr;
    L.a.row_offset = 0;
    memset(&L.a.stage, 0, sizeof L.a.stage);
    if (L.a.priv && L.a.n < PRIV_MIN_ROWS) L.a.priv = 0;
    L.smem = qm_scan_smem_bytes(g.ex.local_slots, g.ex.local_hash, g.pl.agg.n_words, 0, 0, L.a.priv);
    L.blocks = scan_blocks(ctx, L.smem, L.a.n, false);
  }
  const int k = std::min(n, 16);
  while ((int)b->side.size() < k) {
    cudaStream_t s2;
    cudaEvent_t ev;
    CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->side.push_back(s2);
    b->side_ev.push_back(ev);
  }
  if (!b->fork_ev) CK(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
  if (!b->copy_stream) CK(cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking));
  if (!b->ev_start) CK(cudaEventCreate(&b->ev_start));
  if (!b->ev_end) CK(cudaEventCreate(&b->ev_end));
  drop_graph(b);
  return QM_OK;
}

// Issue one wave's device work on stream st: clear its tables and bitmaps,
// scan its queries, rank / lay out / emit / pack their results and copy its
// layout and statuses to pinned host memory.
int wave_launch(qm_batch *b, BatchWave &wv, cudaStream_t st) {
  qm_ctx *ctx = b->ctx;
  if (b->mode == 0) {
    const qm_batch_dev &d = wv.dev;
    CK(qm_batch_launch_init(d, st));
    const int k = std::min<int>((int)wv.classes.size(), (int)b->side.size());
    if (k > 1) {
      CK(cudaEventRecord(b->fork_ev, st));
      for (int j = 0; j < k; j++) CK(cudaStreamWaitEvent(b->side[j], b->fork_ev, 0));
    }
    for (size_t c = 0; c < wv.classes.size(); c++) {
      const BatchWave::ClassLaunch &L = wv.classes[c];
      CK(qm_batch_launch_class(L.cls, d.bq, d.chunks + L.chunk0, L.n_chunks, d.counter + c, L.local_bytes,
                               L.blocks, L.smem, k > 1 ? b->side[c % k] : st));
    }
    if (k > 1)
      for (int j = 0; j < k; j++) {
        CK(cudaEventRecord(b->side_ev[j], b->side[j]));
        CK(cudaStreamWaitEvent(st, b->side_ev[j], 0));
      }
    CK(qm_batch_launch_finalize(d, st));
  } else {
    CK(qm_batch_launch_init(wv.dev, st));
    const int nq = wv.q1 - wv.q0;
    const int k = std::min<int>(nq, (int)b->side.size());
    CK(cudaEventRecord(b->fork_ev, st));
    for (int j = 0; j < k; j++) CK(cudaStreamWaitEvent(b->side[j], b->fork_ev, 0));
    for (int j = 0; j < nq; j++) {
      const qm_batch::Launch &L = b->launches[b->order[wv.q0 + j]];
      CK(qm_launch_scan(L.a, L.blocks, L.smem, b->side[j % k]));
    }
    for (int j = 0; j < k; j++) {
      CK(cudaEventRecord(b->side_ev[j], b->side[j]));
      CK(cudaStreamWaitEvent(st, b->side_ev[j], 0));
    }
    CK(qm_batch_launch_finalize(wv.dev, st));
  }
  CK(cudaMemcpyAsync((qm_status *)b->h_status.p + wv.q0, wv.dev.statuses, sizeof(qm_status) * (wv.q1 - wv.q0),
                     cudaMemcpyDeviceToHost, st));
  return QM_OK;
}

// Issue every wave on the batch's stream (each through its captured graph,
// or with plain launches when use_graph is false), each followed by its
// `done` event.  Nothing waits here.
int batch_issue(qm_batch *b, bool use_graph) {
  qm_ctx *ctx = b->ctx;
  cudaStream_t st = b->st();
  CK(cudaEventRecord(b->ev_start, st));
  for (auto &wp : b->waves) {
    BatchWave &wv = *wp;
    if (use_graph) {
      if (!wv.gexec) {
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc = wave_launch(b, wv, st);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc || e != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
          return rc ? rc : set_err(ctx, QM_ERR_CUDA, "capturing the batched launch: %s", cudaGetErrorString(e));
        }
        wv.graph = g;
        CK(cudaGraphInstantiate(&wv.gexec, g, 0));
      }
      CK(cudaGraphLaunch(wv.gexec, st));
    } else {
      int rc = wave_launch(b, wv, st);
      if (rc) return rc;
    }
    CK(cudaEventRecord(wv.done, st));
  }
  return QM_OK;
}

// Query i's result from its wave's packed results in host memory.
// own: the query's own buffer holding just its region (else the wave's
// buffer of every region).
qm_result *batch_result(qm_batch *b, int i, const BatchWave &wv, const qm_status &s, float scan_ms,
                        const std::shared_ptr<SharedPinned> &own = nullptr) {
  const int j = b->pos[i];
  const qm_batch_meta *meta = (const qm_batch_meta *)wv.h_meta.p;
  const qm_bq &qb = b->bq[i];
  const Plan &pl = b->gts[i].pl;
  const int64_t G = meta->groups[j - wv.q0];
  const std::shared_ptr<SharedPinned> &hold = own ? own : wv.host;
  const uint8_t *h = (const uint8_t *)hold->buf.p;
  qm_result *R = new qm_result();
  R->shared = hold;
  R->n_rows = G;
  int64_t off = own ? 0 : meta->base[j - wv.q0];
  for (int k = 0; k < qb.outs.n_out; k++) {
    qm_result::Col c;
    c.name = pl.meta[k].name;
    c.dtype = qb.outs.o[k].dtype;
    c.is_key = pl.meta[k].is_key;
    c.bytes = (size_t)G * qb.width[k];
    c.data = h + off;
    off += ((int64_t)c.bytes + 15) & ~(int64_t)15;
    if (qb.nullable[k]) {
      c.nulls = h + off;
      const size_t nb = (size_t)((G + 7) / 8);
      for (size_t x = 0; x < nb && !c.has_nulls; x++) c.has_nulls = c.nulls[x] != 0;
      off += ((G + 31) / 32 * 4 + 15) & ~(int64_t)15;
    }
    R->cols.push_back(std::move(c));
  }
  R->stats.rows_scanned = b->rows[i];
  R->stats.rows_selected = (int64_t)s.rows_selected;
  R->stats.groups = G;
  R->stats.bytes_scanned = pl.bytes_per_row * b->rows[i];
  R->stats.scan_ms = scan_ms;
  R->stats.strategy = b->gts[i].ex.strategy;
  R->stats.launches = b->mode == 0 ? 8 : 7 + (wv.q1 - wv.q0);
  return R;
}

// A query's device status as a code; overflowed tables and stale column
// statistics are re-run alone (QM_ERR_CAPACITY), where both are repaired.
int status_code(const qm_status &s) {
  if (s.error == 0) return QM_OK;
  return s.error == QM_DEV_OVERFLOW || s.error == QM_DEV_STALE ? QM_ERR_CAPACITY : QM_ERR_CUDA;
}

// Wait for each wave in turn and copy its packed results back on the copy
// stream while later waves still run; then build one result per query.
// With per_query, each query's region is copied by its own copy and
// on_done(i, code, result) is called as soon as that copy has landed (the
// results of one wave complete one by one); otherwise results[i] and
// codes[i] are filled once every copy has landed.
int batch_collect(qm_batch *b, qm_result **results, int *codes, bool per_query = false,
                  const std::function<void(int, int, qm_result *)> &on_done = nullptr) {
  qm_ctx *ctx = b->ctx;
  const int n = b->n;
  if (per_query && (int)b->q_ev.size() < n) {
    while ((int)b->q_ev.size() < n) {
      cudaEvent_t ev;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      b->q_ev.push_back(ev);
    }
  }
  if (per_query) b->q_host.assign(n, nullptr);
  const qm_status *stv = (const qm_status *)b->h_status.p;
  for (auto &wp : b->waves) {
    BatchWave &wv = *wp;
    cudaError_t e = cudaEventSynchronize(wv.done);
    if (e != cudaSuccess) return set_err(ctx, QM_ERR_CUDA, "batched run: %s", cudaGetErrorString(e));
    const qm_batch_meta *meta = (const qm_batch_meta *)wv.h_meta.p;
    const size_t total = (size_t)meta->total;
    CK(cudaStreamWaitEvent(b->copy_stream, wv.done, 0));
    if (!per_query) {
      auto holder = std::make_shared<SharedPinned>();
      holder->pool = ctx->pool;
      if (!ctx->pool->acquire(total + 16, holder->buf)) return set_err(ctx, QM_ERR_OOM, "pinned batch results");
      wv.host = holder;
      if (total)
        CK(cudaMemcpyAsync(holder->buf.p, wv.dev.packed, total, cudaMemcpyDeviceToHost, b->copy_stream));
      continue;
    }
    // one pinned buffer per query: buffers of one query's size class are
    // reused from request to request, where one buffer per batch would need
    // ever larger ones as batches grow (page-locking a new buffer of
    // gigabytes stalls every lane for most of a second)
    for (int j = wv.q0; j < wv.q1; j++) {
      const int64_t base = meta->base[j - wv.q0], bytes = meta->bytes[j - wv.q0];
      auto holder = std::make_shared<SharedPinned>();
      holder->pool = ctx->pool;
      if (!ctx->pool->acquire((size_t)bytes + 16, holder->buf)) return set_err(ctx, QM_ERR_OOM, "pinned request result");
      b->q_host[j] = holder;
      if (bytes > 0)
        CK(cudaMemcpyAsync(holder->buf.p, wv.dev.packed + base, (size_t)bytes, cudaMemcpyDeviceToHost,
                           b->copy_stream));
      CK(cudaEventRecord(b->q_ev[j], b->copy_stream));
    }
  }
  CK(cudaEventRecord(b->ev_end, b->copy_stream));
  if (per_query) {
    for (auto &wp : b->waves) {
      BatchWave &wv = *wp;
      for (int j = wv.q0; j < wv.q1; j++) {
        cudaError_t e = cudaEventSynchronize(b->q_ev[j]);
        if (e != cudaSuccess) return set_err(ctx, QM_ERR_CUDA, "batched results: %s", cudaGetErrorString(e));
        const int i = b->order[j];
        const int code = status_code(stv[j]);
        qm_result *R = code == QM_OK ? batch_result(b, i, wv, stv[j], 0.f, b->q_host[j]) : nullptr;
        b->q_host[j].reset();
        if (results) results[i] = R;
        if (codes) codes[i] = code;
        if (on_done) on_done(i, code, R);
      }
    }
  }
  cudaError_t e = cudaEventSynchronize(b->ev_end);
  if (e != cudaSuccess) return set_err(ctx, QM_ERR_CUDA, "batched results: %s", cudaGetErrorString(e));
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_end);
  b->last_ms = ms;
  if (!per_query) {
    for (int j = 0; j < n; j++) {
      const int i = b->order[j];
      const BatchWave &wv = *b->waves[b->wave_of[j]];
      codes[i] = status_code(stv[j]);
      results[i] = codes[i] == QM_OK ? batch_result(b, i, wv, stv[j], ms) : nullptr;
      if (results[i]) results[i]->stats.device_ms = ms;
    }
  }
  // the results hold the host buffers now (they return to the pool with them)
  for (auto &wp : b->waves) wp->host.reset();
  return QM_OK;
}

void batch_reset(qm_batch *b, int n) {
  b->n = n;
  b->gts.assign(n, GroupTable());
  b->bq.assign(n, qm_bq());
  b->rows.assign(n, 0);
  b->est.assign(n, 1);
  b->tabs.assign(n, nullptr);
  b->ex_plan.assign(n, Exec());
  b->queries.clear();
  b->queries.resize(n);  // null until planned
  b->total_rows = 0;
  b->bytes_scanned = 0;
  drop_graph(b);
}

// Plan query i of the batch over table t and size its group table (the
// batch's arena is laid out later by batch_layout).
int batch_plan_one(qm_batch *b, int i, const qm_table *table, const qm_query *query) {
  qm_ctx *ctx = b->ctx;
  if (!table || !query) return set_err(ctx, QM_ERR_INVALID, "query %d: null table or query", i);
  if (query->order_by || query->has_limit || query->offset)
    return set_err(ctx, QM_ERR_UNSUPPORTED, "query %d: ORDER BY / LIMIT / OFFSET run through qm_query_run", i);
  b->tabs[i] = table;
  b->queries[i].reset(new OwnedQuery());
  b->queries[i]->copy(*query);
  qm_query q = *query;
  q.flags &= ~QM_FLAG_UNORDERED;  // the batched finalize always orders by first row
  qm_table *t = const_cast<qm_table *>(table);
  GroupTable &gt = b->gts[i];
  int64_t est = 1, direct_size = 0;
  int rc = plan_table_query(ctx, t, &q, gt, est, direct_size);
  if (rc) return rc;
  // sizes as setup_table, without allocating
  Exec &ex = gt.ex;
  if (gt.pl.key.mode == QK_NONE) {
    ex.n_slots = 1;
  } else if (gt.pl.key.mode == QK_DIRECT) {
    ex.n_slots = direct_size;
  } else {
    int64_t want = std::max<int64_t>(1024, est * 2 + est / 8);
    ex.log2cap = ilog2_ceil(want);
    ex.n_slots = (int64_t)1 << ex.log2cap;
  }
  choose_layout(gt.pl, est, ex, ctx->tuning);
  b->est[i] = est;
  b->ex_plan[i] = ex;
  qm_bq &qb = b->bq[i];
  memset(&qb, 0, sizeof qb);
  qb.outs = gt.pl.outs;
  qb.none = gt.pl.key.mode == QK_NONE;
  for (int k = 0; k < qb.outs.n_out; k++) {
    qb.width[k] = (int32_t)dtype_size(qb.outs.o[k].dtype);
    qb.nullable[k] = gt.pl.meta[k].nullable ? 1 : 0;
  }
  b->rows[i] = t->n_rows;
  b->total_rows += t->n_rows;
  b->bytes_scanned += gt.pl.bytes_per_row * t->n_rows;
  return QM_OK;
}

// Device bytes the batch's group tables, bitmaps and packed results take
// (what batch_layout sizes its buffers to).
int64_t batch_query_bytes(const qm_batch *b, int i) {
  const GroupTable &gt = b->gts[i];
  const qm_bq &q = b->bq[i];
  const int64_t total_slots = gt.ex.n_slots + special_slots(gt.pl.key.mode);
  const int64_t table = total_slots * (1 + gt.pl.agg.n_words) * 8;
  const int64_t gmax = q.none ? 1 : std::min<int64_t>(total_slots, std::max<int64_t>(b->rows[i], 1));
  int64_t res = 0;
  for (int k = 0; k < q.outs.n_out; k++) res += (gmax * q.width[k] + 15) / 16 * 16 + (q.nullable[k] ? 2 * gmax + 64 : 0);
  return table + res + b->rows[i] / 8 * 3 + 4096;
}

}  // namespace

extern "C" {

int qm_batch_create(qm_ctx *ctx, int32_t n, const qm_table *const *tables, const qm_query *const *queries,
                    qm_batch **out) {
  if (!ctx || !out || n <= 0 || !tables || !queries) return set_err(ctx, QM_ERR_INVALID, "qm_batch_create: bad arguments");
  if (n > QM_BATCH_MAX) return set_err(ctx, QM_ERR_UNSUPPORTED, "at most %d queries per batch", QM_BATCH_MAX);
  *out = nullptr;
  cudaSetDevice(ctx->device);
  qm_batch *b = new qm_batch();
  b->ctx = ctx;
  batch_reset(b, n);
  for (int i = 0; i < n; i++) {
    int rc = batch_plan_one(b, i, tables[i], queries[i]);
    if (rc) {
      delete b;
      return rc;
    }
  }
  int rc = batch_layout(b);
  if (rc) {
    delete b;
    return rc;
  }
  *out = b;
  return QM_OK;
}

int qm_batch_set_mode(qm_batch *b, int32_t mode) {
  if (!b || (mode != 0 && mode != 1)) return QM_ERR_INVALID;
  if (b->mode != mode) {
    b->mode = mode;
    drop_graph(b);
  }
  return QM_OK;
}

int qm_batch_set_tuning(qm_batch *b, int32_t chunk_tiles, int32_t local_kb, int32_t blocks_per_sm) {
  if (!b) return QM_ERR_INVALID;
  if (chunk_tiles > 0) b->chunk_tiles = chunk_tiles;
  if (local_kb >= 0) b->local_kb = std::min(local_kb, 160);
  if (blocks_per_sm >= 0) b->bps = blocks_per_sm;
  cudaSetDevice(b->ctx->device);
  // rebuild block-local table choices from the planner's, then re-lay out
  for (int i = 0; i < b->n; i++) choose_layout(b->gts[i].pl, b->est[i], b->gts[i].ex, b->ctx->tuning);
  return batch_layout(b);
}

int qm_batch_set_waves(qm_batch *b, int32_t waves) {
  if (!b || waves < 0) return QM_ERR_INVALID;
  cudaSetDevice(b->ctx->device);
  b->waves_req = waves;
  for (int i = 0; i < b->n; i++) choose_layout(b->gts[i].pl, b->est[i], b->gts[i].ex, b->ctx->tuning);
  return batch_layout(b);
}

int qm_batch_run(qm_batch *b, qm_result **results) {
  if (!b || !results) return QM_ERR_INVALID;
  cudaSetDevice(b->ctx->device);
  std::vector<int> codes(b->n, QM_OK);
  for (int i = 0; i < b->n; i++) results[i] = nullptr;
  int rc = batch_issue(b, true);
  if (!rc) rc = batch_collect(b, results, codes.data());
  if (rc) {
    cudaStreamSynchronize(b->st());
    cudaStreamSynchronize(b->copy_stream);
    for (int k = 0; k < b->n; k++) {
      delete results[k];
      results[k] = nullptr;
    }
    return rc;
  }
  for (int i = 0; i < b->n; i++)
    if (codes[i] == QM_ERR_CAPACITY) {
      // more groups than the batched table was sized for: this query alone,
      // where its table regrows
      codes[i] = qm_query_run(b->ctx, b->tabs[i], &b->queries[i]->q, &results[i]);
    }
  for (int i = 0; i < b->n; i++)
    if (codes[i] != QM_OK) {
      for (int k = 0; k < b->n; k++) {
        delete results[k];
        results[k] = nullptr;
      }
      return set_err(b->ctx, codes[i], "query %d of the batch: device status %d (group estimate too small)", i,
                     ((const qm_status *)b->h_status.p)[b->pos[i]].error);
    }
  return QM_OK;
}

int qm_batch_stats(const qm_batch *b, double *device_ms, int64_t *rows, int64_t *bytes, int32_t *chunks) {
  if (!b) return QM_ERR_INVALID;
  if (device_ms) *device_ms = b->last_ms;
  if (rows) *rows = b->total_rows;
  if (bytes) *bytes = b->bytes_scanned;
  if (chunks) {
    int c = 0;
    for (auto &w : b->waves) c += w->dev.n_chunks;
    *chunks = c;
  }
  return QM_OK;
}

int qm_batch_destroy(qm_batch *b) {
  if (!b) return QM_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->st());
  if (b->copy_stream) cudaStreamSynchronize(b->copy_stream);
  delete b;
  return QM_OK;
}

}  // extern "C"

#include "qm_server.cuh"
#include "qm_parquet.cuh"
