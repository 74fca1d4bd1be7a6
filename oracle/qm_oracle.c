/*
 * qm_oracle.c — CPU restatement of QueryMode's filter -> GROUP BY path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path and the timed CPU baseline; it is never linked into, loaded by or
 * called from the product library (querymode_b200/libqm_gpu.so).
 *
 * The reference cannot be built or run here (its engine is TypeScript plus
 * Zig->WASM; neither node nor zig exists in the image), so this is a
 * line-by-line restatement of the reference's semantics:
 *
 *   predicates   src/decode.ts:478-487 (coerceCompare), :489-541
 *                (matchesFilter), :558-578 (rowPassesFilters)
 *   WASM scan    src/operators.ts:550-666 (wasmFilterNumeric /
 *   semantics    wasmFilterRange: NULL read as 0, int32 threshold ToInt32,
 *                int64 threshold safeBigInt) and wasm/src/wasm/
 *                aggregates.zig:605-914 (filter kernels, inclusive BETWEEN)
 *   group keys   src/types.ts:10-18 (groupKeyFrom; String(v) joined by NUL,
 *                NULL -> sentinel).  String equality of the key parts of
 *                numeric columns is equality of (null flag, value) with
 *                -0 == 0 and every NaN equal, which is how keys compare here.
 *   partial agg  src/partial-agg.ts:63-86 (updatePartialAgg),
 *                :89-95 (updatePartialAggBigInt), :141-166 (feedAggStates),
 *                :197-223 (computePartialAggColumnar)
 *   batch merge  src/operators.ts:1656-1681 (first batch partial is the
 *                accumulator; later batch partials merge into it in batch
 *                order) with src/partial-agg.ts:225-267 (mergeStates)
 *   finalize     src/partial-agg.ts:105-134 (resolveValue), :38-44 (bigAvg),
 *                :306-352 (finalizePartialAgg; rows in Map first-seen order)
 *
 * Float SUM is a sequential double sum within a batch, batch sums added in
 * batch order — exactly the reference's order.  For the 1e-12 checks the
 * oracle also reports, per float SUM/AVG cell, a 113-bit (__float128) sum
 * and the sum of magnitudes.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qm_gpu.h"

typedef __int128 i128;

/* ------------------------------------------------------------------ values */
/* A JS value as seen by coerceCompare: a number, or a bigint.  A bigint that
 * came from BigInt(Math.trunc(x)) of a huge double may not fit in 128 bits;
 * it is kept as HUGE with the sign in `d` (only its sign matters when it is
 * compared against an int64 column value). */
enum { JS_NUM = 0, JS_BIG = 1, JS_HUGE = 2 };
typedef struct {
  int kind;
  double d;
  i128 b;
} jsv;

static jsv js_num(double d) { jsv v; v.kind = JS_NUM; v.d = d; v.b = 0; return v; }
static jsv js_big(i128 b) { jsv v; v.kind = JS_BIG; v.d = 0; v.b = b; return v; }

/* BigInt(Math.trunc(x)) for finite x (src/decode.ts:482-483). */
static jsv js_big_of_trunc(double x) {
  double t = trunc(x);
  if (fabs(t) < 1.0e38) return js_big((i128)t); /* exact: t is an integer < 2^127 */
  jsv v; v.kind = JS_HUGE; v.d = t > 0 ? 1.0 : -1.0; v.b = 0; return v;
}

/* coerceCompare (src/decode.ts:480-485) */
static void coerce(jsv a, jsv b, jsv *oa, jsv *ob) {
  if (a.kind != JS_NUM && b.kind == JS_NUM) {
    *oa = a;
    *ob = isfinite(b.d) ? js_big_of_trunc(b.d) : b;
  } else if (a.kind == JS_NUM && b.kind != JS_NUM) {
    *oa = isfinite(a.d) ? js_big_of_trunc(a.d) : a;
    *ob = b;
  } else {
    *oa = a;
    *ob = b;
  }
}

/* Three-way mathematical comparison for JS relational operators between any
 * two values; returns 2 when unordered (a NaN is involved). */
static int js_order(jsv a, jsv b) {
  if (a.kind == JS_NUM && b.kind == JS_NUM) {
    if (isnan(a.d) || isnan(b.d)) return 2;
    return a.d < b.d ? -1 : (a.d > b.d ? 1 : 0);
  }
  if (a.kind == JS_NUM) { int r = js_order(b, a); return r == 2 ? 2 : -r; }
  /* a is a bigint */
  if (a.kind == JS_HUGE) {
    if (b.kind == JS_NUM && isnan(b.d)) return 2;
    if (b.kind == JS_NUM && isinf(b.d)) return b.d > 0 ? -1 : 1;
    if (b.kind == JS_HUGE && b.d == a.d) return 0; /* not reached on the path */
    return a.d > 0 ? 1 : -1;
  }
  if (b.kind == JS_BIG) return a.b < b.b ? -1 : (a.b > b.b ? 1 : 0);
  if (b.kind == JS_HUGE) return b.d > 0 ? -1 : 1;
  /* bigint vs number */
  if (isnan(b.d)) return 2;
  if (isinf(b.d)) return b.d > 0 ? -1 : 1;
  double fl = floor(b.d);
  if (fl >= 1.0e38) return -1;
  if (fl <= -1.0e38) return 1;
  i128 f = (i128)fl;
  if (a.b < f) return -1;
  if (a.b > f) return 1;
  return (b.d == fl) ? 0 : -1;
}

/* JS strict equality between two coerced values. */
static int js_strict_eq(jsv a, jsv b) {
  if (a.kind == JS_NUM && b.kind == JS_NUM) return a.d == b.d;
  if (a.kind == JS_NUM || b.kind == JS_NUM) return 0; /* different types */
  if (a.kind == JS_BIG && b.kind == JS_BIG) return a.b == b.b;
  return 0;
}

static jsv qmv_to_js(const qm_value *v) {
  return v->kind == QM_VAL_BIGINT ? js_big((i128)v->big) : js_num(v->num);
}

/* --------------------------------------------------------------- columns */
typedef struct {
  const char *name;
  int dtype;
  const void *data;
  const uint8_t *nulls;
} ocol;

static int col_is_null(const ocol *c, int64_t r) {
  return c->nulls && ((c->nulls[r >> 3] >> (r & 7)) & 1);
}

/* Value of a non-null cell as decoded by the reference: int64 -> bigint,
 * int32 / float32 / float64 -> number (src/columnar.ts:752-773). */
static jsv col_js(const ocol *c, int64_t r) {
  switch (c->dtype) {
    case QM_I64: return js_big((i128)((const int64_t *)c->data)[r]);
    case QM_I32: return js_num((double)((const int32_t *)c->data)[r]);
    case QM_F32: return js_num((double)((const float *)c->data)[r]);
    default: return js_num(((const double *)c->data)[r]);
  }
}

/* matchesFilter for a non-null value (src/decode.ts:489-541), numeric ops. */
static int js_matches(jsv val, const qm_filter *f) {
  jsv a, b, lo, hi;
  int o;
  switch (f->op) {
    case QM_OP_EQ: coerce(val, qmv_to_js(&f->value), &a, &b); return js_strict_eq(a, b);
    case QM_OP_NEQ: coerce(val, qmv_to_js(&f->value), &a, &b); return !js_strict_eq(a, b);
    case QM_OP_GT: coerce(val, qmv_to_js(&f->value), &a, &b); o = js_order(a, b); return o == 1;
    case QM_OP_GTE: coerce(val, qmv_to_js(&f->value), &a, &b); o = js_order(a, b); return o == 1 || o == 0;
    case QM_OP_LT: coerce(val, qmv_to_js(&f->value), &a, &b); o = js_order(a, b); return o == -1;
    case QM_OP_LTE: coerce(val, qmv_to_js(&f->value), &a, &b); o = js_order(a, b); return o == -1 || o == 0;
    case QM_OP_BETWEEN: {
      jsv t;
      coerce(val, qmv_to_js(&f->value), &t, &lo);
      coerce(val, qmv_to_js(&f->value2), &a, &hi);
      int o1 = js_order(a, lo), o2 = js_order(a, hi);
      return (o1 == 1 || o1 == 0) && (o2 == -1 || o2 == 0);
    }
    case QM_OP_NOT_BETWEEN: {
      jsv t;
      coerce(val, qmv_to_js(&f->value), &t, &lo);
      coerce(val, qmv_to_js(&f->value2), &a, &hi);
      int o1 = js_order(a, lo), o2 = js_order(a, hi);
      return o1 == -1 || o2 == 1;
    }
    default: return 1; /* src/decode.ts:551 default: true */
  }
}

/* rowPassesFilters' per-filter test (src/decode.ts:559-564). */
static int js_filter_row(const ocol *c, int64_t r, const qm_filter *f) {
  int isnull = col_is_null(c, r);
  if (f->op == QM_OP_IS_NULL) return isnull;
  if (f->op == QM_OP_IS_NOT_NULL) return !isnull;
  if (isnull) return 0;
  return js_matches(col_js(c, r), f);
}

/* ECMAScript ToInt32 (JS number -> WASM i32 parameter). */
static int32_t to_int32(double x) {
  if (!isfinite(x)) return 0;
  double t = trunc(x);
  double m = fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  uint32_t u = (uint32_t)m;
  return (int32_t)u;
}

/* safeBigInt then ToBigInt64 (JS bigint -> WASM i64 parameter wraps mod 2^64). */
static int64_t to_wasm_i64(double x) {
  if (!isfinite(x)) return 0;
  double t = trunc(x);
  if (fabs(t) < 9.2e18) return (int64_t)t;
  /* exact modular reduction of a huge integer-valued double */
  double m = fmod(t, 18446744073709551616.0);
  if (m < 0) m += 18446744073709551616.0;
  uint64_t u = m >= 9223372036854775808.0 ? (uint64_t)(m - 9223372036854775808.0) + 9223372036854775808ULL
                                           : (uint64_t)m;
  return (int64_t)u;
}

static int cmp_op_i64(int64_t v, int op, int64_t t) {
  switch (op) {
    case 0: return v == t; case 1: return v != t; case 2: return v < t;
    case 3: return v <= t; case 4: return v > t; default: return v >= t;
  }
}
static int cmp_op_f64(double v, int op, double t) {
  switch (op) {
    case 0: return v == t; case 1: return v != t; case 2: return v < t;
    case 3: return v <= t; case 4: return v > t; default: return v >= t;
  }
}

/* Does the WASM scan route (applyAndFilters, src/operators.ts:469-547) take
 * its WASM branch for this filter?  Returns 0 when it falls back to JS. */
static int wasm_route(const ocol *c, const qm_filter *f) {
  if (f->op <= QM_OP_GTE) {
    if (f->value.kind != QM_VAL_NUMBER) return 0;
    if (c->dtype == QM_I64 && !isfinite(f->value.num)) return 0; /* :586 */
    return 1;
  }
  if (f->op == QM_OP_BETWEEN || f->op == QM_OP_NOT_BETWEEN) {
    if (f->value.kind != QM_VAL_NUMBER || f->value2.kind != QM_VAL_NUMBER) return 0;
    if (c->dtype == QM_I64 && (!isfinite(f->value.num) || !isfinite(f->value2.num))) return 0; /* :639 */
    return 1;
  }
  return 0;
}

/* WASM filter kernels over a page copied with NULL -> 0
 * (src/operators.ts:562-605, wasm/src/wasm/aggregates.zig:605-914). */
static int wasm_filter_row(const ocol *c, int64_t r, const qm_filter *f) {
  int isnull = col_is_null(c, r);
  int range = f->op == QM_OP_BETWEEN || f->op == QM_OP_NOT_BETWEEN;
  int neg = f->op == QM_OP_NOT_BETWEEN;
  if (c->dtype == QM_F64 || c->dtype == QM_F32) {
    double v = isnull ? 0.0 : (c->dtype == QM_F64 ? ((const double *)c->data)[r]
                                                 : (double)((const float *)c->data)[r]);
    if (!range) return cmp_op_f64(v, f->op, f->value.num);
    double lo = f->value.num, hi = f->value2.num;
    return neg ? (v < lo || v > hi) : (v >= lo && v <= hi);
  }
  if (c->dtype == QM_I32) {
    int32_t v = isnull ? 0 : ((const int32_t *)c->data)[r];
    if (!range) return cmp_op_i64(v, f->op, to_int32(f->value.num));
    int32_t lo = to_int32(f->value.num), hi = to_int32(f->value2.num);
    return neg ? (v < lo || v > hi) : (v >= lo && v <= hi);
  }
  int64_t v = isnull ? 0 : ((const int64_t *)c->data)[r];
  if (!range) return cmp_op_i64(v, f->op, to_wasm_i64(f->value.num));
  int64_t lo = to_wasm_i64(f->value.num), hi = to_wasm_i64(f->value2.num);
  return neg ? (v < lo || v > hi) : (v >= lo && v <= hi);
}

typedef struct {
  const qm_filter *f;
  const ocol *c;
  int wasm;
} oterm;

static int term_pass(const oterm *t, int64_t r) {
  return t->wasm ? wasm_filter_row(t->c, r, t->f) : js_filter_row(t->c, r, t->f);
}

/* ------------------------------------------------------------ group map */
#define OR_MAX_KEYS 4

typedef struct {
  double sum;
  int64_t count;
  double min, max;
  int has_big;
  i128 bigsum;
  int64_t bigmin, bigmax;
  /* diagnostics for the float-sum tolerance checks */
  __float128 xsum;
  double abssum;
} ostate;

typedef struct {
  int n_keys;
  int n_aggs;
  int64_t cap;      /* power of two */
  int64_t n_groups;
  int64_t *slot;    /* cap entries: group index or -1 */
  uint64_t *keys;   /* n_groups x n_keys normalized values */
  uint8_t *knull;   /* n_groups x n_keys */
  ostate *st;       /* n_groups x n_aggs */
  int64_t alloc_groups;
} omap;

static uint64_t fmix64(uint64_t k) {
  k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL; k ^= k >> 33; return k;
}

static void omap_init(omap *m, int n_keys, int n_aggs) {
  memset(m, 0, sizeof(*m));
  m->n_keys = n_keys; m->n_aggs = n_aggs; m->cap = 64;
  m->slot = (int64_t *)malloc(sizeof(int64_t) * m->cap);
  for (int64_t i = 0; i < m->cap; i++) m->slot[i] = -1;
  m->alloc_groups = 32;
  m->keys = (uint64_t *)malloc(sizeof(uint64_t) * m->alloc_groups * (n_keys ? n_keys : 1));
  m->knull = (uint8_t *)malloc(m->alloc_groups * (n_keys ? n_keys : 1));
  m->st = (ostate *)malloc(sizeof(ostate) * m->alloc_groups * (n_aggs ? n_aggs : 1));
}

static void omap_free(omap *m) {
  free(m->slot); free(m->keys); free(m->knull); free(m->st);
  memset(m, 0, sizeof(*m));
}

static uint64_t key_hash(const uint64_t *k, const uint8_t *kn, int n) {
  uint64_t h = 0x9e3779b97f4a7c15ULL;
  for (int i = 0; i < n; i++) h = fmix64(h ^ (kn[i] ? 0x5bd1e995ULL : k[i]) ^ ((uint64_t)i << 56));
  return h;
}

static void omap_grow(omap *m) {
  int64_t ncap = m->cap * 2;
  int64_t *ns = (int64_t *)malloc(sizeof(int64_t) * ncap);
  for (int64_t i = 0; i < ncap; i++) ns[i] = -1;
  for (int64_t g = 0; g < m->n_groups; g++) {
    uint64_t h = key_hash(m->keys + g * m->n_keys, m->knull + g * m->n_keys, m->n_keys);
    int64_t s = (int64_t)(h & (uint64_t)(ncap - 1));
    while (ns[s] >= 0) s = (s + 1) & (ncap - 1);
    ns[s] = g;
  }
  free(m->slot); m->slot = ns; m->cap = ncap;
}

/* initPartialAggState (src/partial-agg.ts:46-61): sum 0, count 0,
 * min Infinity, max -Infinity. */
static void ostate_init(ostate *s) {
  memset(s, 0, sizeof(*s));
  s->min = INFINITY; s->max = -INFINITY;
}

/* Map.get / Map.set on the group key (src/partial-agg.ts:217-219). */
static int64_t omap_find_or_add(omap *m, const uint64_t *k, const uint8_t *kn) {
  uint64_t h = key_hash(k, kn, m->n_keys);
  int64_t s = (int64_t)(h & (uint64_t)(m->cap - 1));
  for (;;) {
    int64_t g = m->slot[s];
    if (g < 0) break;
    if (memcmp(m->keys + g * m->n_keys, k, sizeof(uint64_t) * m->n_keys) == 0 &&
        memcmp(m->knull + g * m->n_keys, kn, m->n_keys) == 0)
      return g;
    s = (s + 1) & (m->cap - 1);
  }
  if (m->n_groups == m->alloc_groups) {
    m->alloc_groups *= 2;
    int nk = m->n_keys ? m->n_keys : 1, na = m->n_aggs ? m->n_aggs : 1;
    m->keys = (uint64_t *)realloc(m->keys, sizeof(uint64_t) * m->alloc_groups * nk);
    m->knull = (uint8_t *)realloc(m->knull, m->alloc_groups * nk);
    m->st = (ostate *)realloc(m->st, sizeof(ostate) * m->alloc_groups * na);
  }
  int64_t g = m->n_groups++;
  memcpy(m->keys + g * m->n_keys, k, sizeof(uint64_t) * m->n_keys);
  memcpy(m->knull + g * m->n_keys, kn, m->n_keys);
  for (int a = 0; a < m->n_aggs; a++) ostate_init(&m->st[g * m->n_aggs + a]);
  m->slot[s] = g;
  if (m->n_groups * 2 > m->cap) omap_grow(m);
  return g;
}

/* Normalized key part: the String(v) identity of a numeric cell. */
static void key_part(const ocol *c, int64_t r, uint64_t *k, uint8_t *kn) {
  if (col_is_null(c, r)) { *k = 0; *kn = 1; return; }
  *kn = 0;
  switch (c->dtype) {
    case QM_I64: *k = (uint64_t)((const int64_t *)c->data)[r]; return;
    case QM_I32: *k = (uint64_t)(int64_t)((const int32_t *)c->data)[r]; return;
    default: {
      double d = c->dtype == QM_F64 ? ((const double *)c->data)[r] : (double)((const float *)c->data)[r];
      if (d == 0.0) d = 0.0;                  /* String(-0) === "0" */
      if (isnan(d)) { *k = 0x7ff8000000000000ULL; return; } /* "NaN" */
      memcpy(k, &d, 8);
      return;
    }
  }
}

/* ------------------------------------------------------------ aggregates */
typedef struct {
  int fn;
  int star;        /* column "*" */
  const ocol *c;
} oagg;

/* updatePartialAgg (number) / updatePartialAggBigInt (bigint), as chosen by
 * feedAggStates (src/partial-agg.ts:141-166). */
static void feed(ostate *s, const oagg *a, int64_t r) {
  if (a->star) { s->count++; return; }
  if (col_is_null(a->c, r)) return; /* null/undefined: skipped */
  if (a->c->dtype == QM_I64) {
    int64_t v = ((const int64_t *)a->c->data)[r];
    s->bigsum = (s->has_big ? s->bigsum : 0) + (i128)v;
    s->count++;
    if (!s->has_big || v < s->bigmin) s->bigmin = v;
    if (!s->has_big || v > s->bigmax) s->bigmax = v;
    s->has_big = 1;
    return;
  }
  double v = col_js(a->c, r).d;
  s->sum += v;
  s->count++;
  if (v < s->min) s->min = v;
  if (v > s->max) s->max = v;
  s->xsum += (__float128)v;
  s->abssum += fabs(v);
}

/* mergeStates (src/partial-agg.ts:225-267), numeric fields. */
static void merge_state(ostate *t, const ostate *s) {
  t->sum += s->sum;
  t->count += s->count;
  if (s->min < t->min) t->min = s->min;
  if (s->max > t->max) t->max = s->max;
  if (s->has_big) {
    t->bigsum = (t->has_big ? t->bigsum : 0) + s->bigsum;
    if (!t->has_big || s->bigmin < t->bigmin) t->bigmin = s->bigmin;
    if (!t->has_big || s->bigmax > t->bigmax) t->bigmax = s->bigmax;
    t->has_big = 1;
  }
  t->xsum += s->xsum;
  t->abssum += s->abssum;
}

/* ------------------------------------------------------------- results */
typedef struct {
  char *name;
  int dtype;
  int is_key;
  void *data;
  uint8_t *nulls;
  int any_null;
  /* diagnostics (float SUM / AVG only) */
  double *xsum_hi, *xsum_lo, *abssum;
} ocolout;

typedef struct {
  int64_t n_rows;
  int n_cols;
  ocolout *cols;
} oresult;

static char *dupstr(const char *s) {
  size_t n = strlen(s);
  char *d = (char *)malloc(n + 1);
  memcpy(d, s, n + 1);
  return d;
}

/* Number(bigint) — round to nearest, ties to even. */
static double i128_to_double(i128 x) {
  int neg = x < 0;
  unsigned __int128 u = neg ? (unsigned __int128)(-(x + 1)) + 1 : (unsigned __int128)x;
  uint64_t hi = (uint64_t)(u >> 64), lo = (uint64_t)u;
  double r;
  if (hi == 0) {
    r = (double)lo; /* correctly rounded u64 -> double conversion */
  } else {
    int lz = __builtin_clzll(hi);
    int shift = 64 - lz;           /* bits to drop so the value fits 64 bits */
    unsigned __int128 mask = (((unsigned __int128)1) << shift) - 1;
    uint64_t top = (uint64_t)(u >> shift);
    int sticky = (u & mask) != 0;
    /* top has 64 significant bits: keep 53, round with guard/sticky */
    uint64_t keep = top >> 11, rem = top & 0x7ff;
    int st = sticky || (rem & 0x3ff);
    int guard = (rem >> 10) & 1;
    if (guard && (st || (keep & 1))) keep++;
    r = ldexp((double)keep, shift + 11);
  }
  return neg ? -r : r;
}

/* bigAvg (src/partial-agg.ts:38-44) with numSum == 0. */
static double big_avg(i128 sum, int64_t count) {
  i128 q = sum / (i128)count, rm = sum % (i128)count;
  double quotient = i128_to_double(q);
  double remainder = i128_to_double(rm);
  return quotient + (remainder + 0.0) / (double)count;
}

static int result_dtype(const oagg *a) {
  if (a->fn == QM_AGG_COUNT) return QM_I64;
  if (a->fn == QM_AGG_AVG) return QM_F64;
  int d = a->c->dtype;
  if (a->fn == QM_AGG_SUM) return d == QM_I64 ? QM_I128 : QM_F64;
  /* MIN / MAX */
  if (d == QM_I64) return QM_I64;
  if (d == QM_I32) return QM_I32;
  return QM_F64;
}

static int dtype_size(int d) {
  return d == QM_I32 || d == QM_F32 ? 4 : (d == QM_I128 ? 16 : 8);
}

/* ------------------------------------------------------------- driver */
typedef struct {
  int64_t n_rows;
  int n_cols;
  ocol *cols;
  int wasm;
  int n_and, n_or_total;
  oterm *and_t, *or_t;
  const qm_query *q;
  int nk, na;
  const ocol *kc[OR_MAX_KEYS];
  oagg *ag;
} oplan;

static const ocol *find_col(const oplan *t, const char *name) {
  for (int i = 0; i < t->n_cols; i++)
    if (strcmp(t->cols[i].name, name) == 0) return &t->cols[i];
  return NULL;
}

static char g_err[512];
const char *oracle_last_error(void) { return g_err; }

static void plan_free(oplan *P) {
  free(P->and_t); free(P->or_t); free(P->cols); free(P->ag);
  memset(P, 0, sizeof(*P));
}

static int plan_build(oplan *P, int64_t n_rows, int32_t n_cols, const qm_column *cols,
                      const qm_query *q, int need_aggs) {
  memset(P, 0, sizeof(*P));
  P->n_rows = n_rows; P->n_cols = n_cols; P->q = q;
  P->cols = (ocol *)calloc(n_cols ? n_cols : 1, sizeof(ocol));
  for (int i = 0; i < n_cols; i++) {
    P->cols[i].name = cols[i].name; P->cols[i].dtype = cols[i].dtype;
    P->cols[i].data = cols[i].data; P->cols[i].nulls = cols[i].null_bitmap;
  }
  P->wasm = (q->flags & QM_FLAG_WASM_SCAN_SEMANTICS) != 0;
  P->n_and = q->n_filters;
  for (int g = 0; g < q->n_or_groups; g++) P->n_or_total += q->or_group_sizes[g];
  P->and_t = (oterm *)calloc(P->n_and + 1, sizeof(oterm));
  P->or_t = (oterm *)calloc(P->n_or_total + 1, sizeof(oterm));
  P->ag = (oagg *)calloc(q->n_aggregates + 1, sizeof(oagg));
  for (int i = 0; i < P->n_and; i++) {
    P->and_t[i].f = &q->filters[i];
    P->and_t[i].c = find_col(P, q->filters[i].column);
    if (!P->and_t[i].c) { snprintf(g_err, sizeof g_err, "unknown filter column %s", q->filters[i].column); return QM_ERR_NOT_FOUND; }
    P->and_t[i].wasm = P->wasm && wasm_route(P->and_t[i].c, P->and_t[i].f);
  }
  for (int i = 0; i < P->n_or_total; i++) {
    P->or_t[i].f = &q->or_filters[i];
    P->or_t[i].c = find_col(P, q->or_filters[i].column);
    if (!P->or_t[i].c) { snprintf(g_err, sizeof g_err, "unknown filter column %s", q->or_filters[i].column); return QM_ERR_NOT_FOUND; }
    P->or_t[i].wasm = P->wasm && wasm_route(P->or_t[i].c, P->or_t[i].f);
  }
  if (!need_aggs) return 0;
  P->nk = q->n_group_by; P->na = q->n_aggregates;
  if (P->nk > OR_MAX_KEYS) { snprintf(g_err, sizeof g_err, "too many group columns"); return QM_ERR_UNSUPPORTED; }
  for (int i = 0; i < P->nk; i++) {
    P->kc[i] = find_col(P, q->group_by[i]);
    if (!P->kc[i]) { snprintf(g_err, sizeof g_err, "unknown group column %s", q->group_by[i]); return QM_ERR_NOT_FOUND; }
  }
  for (int i = 0; i < P->na; i++) {
    P->ag[i].fn = q->aggregates[i].fn;
    P->ag[i].star = strcmp(q->aggregates[i].column, "*") == 0;
    if (!P->ag[i].star) {
      P->ag[i].c = find_col(P, q->aggregates[i].column);
      if (!P->ag[i].c) { snprintf(g_err, sizeof g_err, "unknown aggregate column %s", q->aggregates[i].column); return QM_ERR_NOT_FOUND; }
    } else if (P->ag[i].fn != QM_AGG_COUNT) {
      snprintf(g_err, sizeof g_err, "only COUNT takes *"); return QM_ERR_INVALID;
    }
  }
  return 0;
}

/* rowPassesFilters over AND filters plus OR groups (src/decode.ts:558-578). */
static int row_pass(const oplan *P, int64_t r) {
  for (int i = 0; i < P->n_and; i++) if (!term_pass(&P->and_t[i], r)) return 0;
  if (P->q->n_or_groups > 0) {
    int off = 0;
    for (int g = 0; g < P->q->n_or_groups; g++) {
      int all = 1;
      for (int i = 0; i < P->q->or_group_sizes[g] && all; i++) all = term_pass(&P->or_t[off + i], r);
      if (all) return 1;
      off += P->q->or_group_sizes[g];
    }
    return 0;
  }
  return 1;
}

/* Aggregate batches [b_lo, b_hi) of `batch_rows` rows into *acc, merging
 * each batch partial into the accumulator in batch order
 * (AggregateOperator.next, src/operators.ts:1656-1681). */
static void process_batches(const oplan *P, int64_t batch_rows, int64_t b_lo, int64_t b_hi,
                            omap *acc, int *have_acc) {
  int nk = P->nk, na = P->na;
  omap part;
  omap_init(&part, nk, na);
  uint64_t kv[OR_MAX_KEYS] = {0};
  uint8_t kn[OR_MAX_KEYS] = {0};
  for (int64_t b = b_lo; b < b_hi; b++) {
    int64_t r0 = b * batch_rows, r1 = r0 + batch_rows < P->n_rows ? r0 + batch_rows : P->n_rows;
    omap_free(&part);
    omap_init(&part, nk, na);
    for (int64_t r = r0; r < r1; r++) {
      if (!row_pass(P, r)) continue;
      for (int i = 0; i < nk; i++) key_part(P->kc[i], r, &kv[i], &kn[i]);
      int64_t g = omap_find_or_add(&part, kv, kn);
      for (int a = 0; a < na; a++) feed(&part.st[g * na + a], &P->ag[a], r);
    }
    if (!*have_acc) {
      omap_free(acc);
      *acc = part;
      omap_init(&part, nk, na);
      *have_acc = 1;
    } else {
      for (int64_t g = 0; g < part.n_groups; g++) {
        int64_t t = omap_find_or_add(acc, part.keys + g * nk, part.knull + g * nk);
        for (int a = 0; a < na; a++) merge_state(&acc->st[t * na + a], &part.st[g * na + a]);
      }
    }
  }
  omap_free(&part);
}

/* merge map `src` into `dst` in src's first-seen order */
static void merge_maps(const oplan *P, omap *dst, const omap *src) {
  for (int64_t g = 0; g < src->n_groups; g++) {
    int64_t t = omap_find_or_add(dst, src->keys + g * P->nk, src->knull + g * P->nk);
    for (int a = 0; a < P->na; a++) merge_state(&dst->st[t * P->na + a], &src->st[g * P->na + a]);
  }
}

/* finalizePartialAgg (src/partial-agg.ts:306-352) */
static oresult *finalize(const oplan *P, omap *acc) {
  const qm_query *q = P->q;
  int nk = P->nk, na = P->na;
  oresult *R = (oresult *)calloc(1, sizeof(oresult));
  int64_t G;
  if (nk == 0) {
    /* ungrouped: exactly one row (src/partial-agg.ts:313-320) */
    if (acc->n_groups == 0) { uint64_t kv[1] = {0}; uint8_t kn[1] = {0}; omap_find_or_add(acc, kv, kn); }
    G = 1;
  } else {
    G = acc->n_groups;
  }
  R->n_rows = G;
  R->n_cols = nk + na;
  R->cols = (ocolout *)calloc(R->n_cols ? R->n_cols : 1, sizeof(ocolout));
  for (int i = 0; i < nk; i++) {
    ocolout *o = &R->cols[i];
    o->name = dupstr(q->group_by[i]);
    o->dtype = P->kc[i]->dtype == QM_F32 ? QM_F64 : P->kc[i]->dtype;
    o->is_key = 1;
    o->data = calloc(G ? G : 1, dtype_size(o->dtype));
    o->nulls = (uint8_t *)calloc((G + 7) / 8 + 1, 1);
    for (int64_t g = 0; g < G; g++) {
      uint64_t k = acc->keys[g * nk + i];
      if (acc->knull[g * nk + i]) { o->nulls[g >> 3] |= (uint8_t)(1u << (g & 7)); o->any_null = 1; continue; }
      if (o->dtype == QM_I32) ((int32_t *)o->data)[g] = (int32_t)(int64_t)k;
      else memcpy((char *)o->data + 8 * g, &k, 8);
    }
  }
  for (int a = 0; a < na; a++) {
    ocolout *o = &R->cols[nk + a];
    const qm_aggregate *qa = &q->aggregates[a];
    if (qa->alias) o->name = dupstr(qa->alias);
    else {
      static const char *fnn[] = {"sum", "avg", "min", "max", "count"};
      size_t n = strlen(fnn[qa->fn]) + 1 + strlen(qa->column) + 1;
      o->name = (char *)malloc(n);
      snprintf(o->name, n, "%s_%s", fnn[qa->fn], qa->column);
    }
    o->dtype = result_dtype(&P->ag[a]);
    o->data = calloc(G ? G : 1, dtype_size(o->dtype));
    o->nulls = (uint8_t *)calloc((G + 7) / 8 + 1, 1);
    int fsum = !P->ag[a].star && (qa->fn == QM_AGG_SUM || qa->fn == QM_AGG_AVG) && P->ag[a].c->dtype != QM_I64;
    if (fsum) {
      o->xsum_hi = (double *)calloc(G ? G : 1, 8);
      o->xsum_lo = (double *)calloc(G ? G : 1, 8);
      o->abssum = (double *)calloc(G ? G : 1, 8);
    }
    for (int64_t g = 0; g < G; g++) {
      ostate *s = &acc->st[g * na + a];
      if (fsum) {
        /* AVG cells carry the exact mean and the mean magnitude instead */
        __float128 x = s->xsum;
        double ab = s->abssum;
        if (qa->fn == QM_AGG_AVG && s->count > 0) { x = x / (__float128)s->count; ab = ab / (double)s->count; }
        o->xsum_hi[g] = (double)x;
        o->xsum_lo[g] = (double)(x - (__float128)o->xsum_hi[g]);
        o->abssum[g] = ab;
      }
      /* resolveValue (src/partial-agg.ts:105-134) */
      if (qa->fn == QM_AGG_COUNT) { ((int64_t *)o->data)[g] = s->count; continue; }
      if (s->count == 0) { o->nulls[g >> 3] |= (uint8_t)(1u << (g & 7)); o->any_null = 1; continue; }
      switch (qa->fn) {
        case QM_AGG_SUM:
          if (s->has_big) { i128 v = s->bigsum; memcpy((char *)o->data + 16 * g, &v, 16); }
          else ((double *)o->data)[g] = s->sum;
          break;
        case QM_AGG_AVG:
          ((double *)o->data)[g] = s->has_big ? big_avg(s->bigsum, s->count) : s->sum / (double)s->count;
          break;
        case QM_AGG_MIN:
        case QM_AGG_MAX: {
          int mx = qa->fn == QM_AGG_MAX;
          if (s->has_big) ((int64_t *)o->data)[g] = mx ? s->bigmax : s->bigmin;
          else if (o->dtype == QM_I32) ((int32_t *)o->data)[g] = (int32_t)(mx ? s->max : s->min);
          else ((double *)o->data)[g] = mx ? s->max : s->min;
          break;
        }
      }
    }
  }
  return R;
}

/* Runs the query.  batch_rows <= 0 means one batch (the in-memory route of
 * MaterializedExecutor, src/client.ts:1023-1054).  Returns 0 or a QM_ERR. */
int oracle_run(int64_t n_rows, int32_t n_cols, const qm_column *cols,
               const qm_query *q, int64_t batch_rows, oresult **out) {
  *out = NULL;
  g_err[0] = 0;
  oplan P;
  int rc = plan_build(&P, n_rows, n_cols, cols, q, 1);
  if (rc) { plan_free(&P); return rc; }
  if (batch_rows <= 0) batch_rows = n_rows > 0 ? n_rows : 1;
  int64_t nb = (n_rows + batch_rows - 1) / batch_rows;
  omap acc;
  int have = 0;
  omap_init(&acc, P.nk, P.na);
  process_batches(&P, batch_rows, 0, nb, &acc, &have);
  *out = finalize(&P, &acc);
  omap_free(&acc);
  plan_free(&P);
  return 0;
}

typedef struct {
  const oplan *P;
  int64_t batch_rows, b_lo, b_hi;
  omap acc;
  int have;
} oworker;

static void *worker_main(void *arg) {
  oworker *w = (oworker *)arg;
  process_batches(w->P, w->batch_rows, w->b_lo, w->b_hi, &w->acc, &w->have);
  return NULL;
}

/* The same query on n_threads host threads: each thread aggregates a
 * contiguous run of batches, and the per-thread partials are merged in
 * thread order — the reference's fragment fan-out and partial merge
 * (src/query-do.ts:1747-1887, src/merge.ts:156-172).  Float sums are then
 * associated per thread rather than strictly per batch.  Used to time the
 * CPU baseline on all host cores. */
int oracle_run_mt(int64_t n_rows, int32_t n_cols, const qm_column *cols,
                  const qm_query *q, int64_t batch_rows, int32_t n_threads,
                  oresult **out) {
  *out = NULL;
  g_err[0] = 0;
  oplan P;
  int rc = plan_build(&P, n_rows, n_cols, cols, q, 1);
  if (rc) { plan_free(&P); return rc; }
  if (batch_rows <= 0) batch_rows = 65536;
  int64_t nb = (n_rows + batch_rows - 1) / batch_rows;
  if (n_threads < 1) n_threads = 1;
  if (n_threads > nb) n_threads = nb > 0 ? (int32_t)nb : 1;
  oworker *W = (oworker *)calloc(n_threads, sizeof(oworker));
  pthread_t *th = (pthread_t *)calloc(n_threads, sizeof(pthread_t));
  for (int t = 0; t < n_threads; t++) {
    W[t].P = &P; W[t].batch_rows = batch_rows;
    W[t].b_lo = nb * t / n_threads; W[t].b_hi = nb * (t + 1) / n_threads;
    omap_init(&W[t].acc, P.nk, P.na);
    pthread_create(&th[t], NULL, worker_main, &W[t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  omap acc;
  omap_init(&acc, P.nk, P.na);
  for (int t = 0; t < n_threads; t++) {
    if (W[t].have) merge_maps(&P, &acc, &W[t].acc);
    omap_free(&W[t].acc);
  }
  *out = finalize(&P, &acc);
  omap_free(&acc);
  free(W); free(th);
  plan_free(&P);
  return 0;
}

/* ------------------------------------------------ key-partitioned threads */
/* One batch over all rows (the in-memory route of MaterializedExecutor,
 * src/client.ts:1023-1054) on n_threads host threads, with the single-thread
 * result bit for bit: thread t takes the groups whose key hash falls in its
 * part, visiting their rows in row order, so every group's float sum is the
 * reference's sequential sum in row order.  The groups of all parts are then
 * put in first-seen order (the Map insertion order of finalizePartialAgg,
 * src/partial-agg.ts:320-349) by a merge on each group's first row.  For
 * full-size checks of high-cardinality results, where merging per-thread
 * maps of millions of groups would dominate. */
typedef struct {
  const oplan *P;
  int part, n_parts;
  uint8_t *row_part;  /* per row: its group's part, or 0xff when filtered out */
  int64_t r0, r1;     /* rows this thread classifies */
  omap acc;
  int64_t *first;   /* first row of each group of acc */
  int64_t n_first, cap_first;
} okworker;

/* Phase 1, by row ranges: the filter, and each passing row's part. */
static void *keypart_classify(void *arg) {
  okworker *w = (okworker *)arg;
  const oplan *P = w->P;
  const int nk = P->nk;
  uint64_t kv[OR_MAX_KEYS] = {0};
  uint8_t kn[OR_MAX_KEYS] = {0};
  for (int64_t r = w->r0; r < w->r1; r++) {
    if (!row_pass(P, r)) {
      w->row_part[r] = 0xff;
      continue;
    }
    for (int i = 0; i < nk; i++) key_part(P->kc[i], r, &kv[i], &kn[i]);
    w->row_part[r] = (uint8_t)((key_hash(kv, kn, nk) >> 40) % (uint64_t)w->n_parts);
  }
  return NULL;
}

/* Phase 2, by part: the part's rows aggregated in row order. */
static void *keypart_main(void *arg) {
  okworker *w = (okworker *)arg;
  const oplan *P = w->P;
  const int nk = P->nk, na = P->na;
  uint64_t kv[OR_MAX_KEYS] = {0};
  uint8_t kn[OR_MAX_KEYS] = {0};
  const uint8_t me = (uint8_t)w->part;
  for (int64_t r = 0; r < P->n_rows; r++) {
    if (w->row_part[r] != me) continue;
    for (int i = 0; i < nk; i++) key_part(P->kc[i], r, &kv[i], &kn[i]);
    const int64_t before = w->acc.n_groups;
    int64_t g = omap_find_or_add(&w->acc, kv, kn);
    if (w->acc.n_groups != before) {
      if (w->n_first == w->cap_first) {
        w->cap_first = w->cap_first ? 2 * w->cap_first : 1024;
        w->first = (int64_t *)realloc(w->first, sizeof(int64_t) * w->cap_first);
      }
      w->first[w->n_first++] = r;
    }
    for (int a = 0; a < na; a++) feed(&w->acc.st[g * na + a], &P->ag[a], r);
  }
  return NULL;
}

int oracle_run_keypart(int64_t n_rows, int32_t n_cols, const qm_column *cols, const qm_query *q,
                       int32_t n_threads, oresult **out) {
  *out = NULL;
  g_err[0] = 0;
  if (q->n_group_by == 0 || n_threads <= 1) return oracle_run(n_rows, n_cols, cols, q, 0, out);
  oplan P;
  int rc = plan_build(&P, n_rows, n_cols, cols, q, 1);
  if (rc) { plan_free(&P); return rc; }
  const int nk = P.nk, na = P.na;
  if (n_threads > 250) n_threads = 250;
  okworker *W = (okworker *)calloc(n_threads, sizeof(okworker));
  pthread_t *th = (pthread_t *)calloc(n_threads, sizeof(pthread_t));
  uint8_t *row_part = (uint8_t *)malloc(n_rows > 0 ? (size_t)n_rows : 1);
  for (int t = 0; t < n_threads; t++) {
    W[t].P = &P; W[t].part = t; W[t].n_parts = n_threads; W[t].row_part = row_part;
    W[t].r0 = n_rows * t / n_threads; W[t].r1 = n_rows * (t + 1) / n_threads;
    pthread_create(&th[t], NULL, keypart_classify, &W[t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  for (int t = 0; t < n_threads; t++) {
    omap_init(&W[t].acc, nk, na);
    pthread_create(&th[t], NULL, keypart_main, &W[t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(row_part);
  /* the parts' groups, each part already in first-row order, merged by first row */
  int64_t G = 0;
  for (int t = 0; t < n_threads; t++) G += W[t].acc.n_groups;
  omap acc;
  memset(&acc, 0, sizeof acc);
  acc.n_keys = nk; acc.n_aggs = na; acc.n_groups = G; acc.alloc_groups = G ? G : 1;
  acc.keys = (uint64_t *)malloc(sizeof(uint64_t) * acc.alloc_groups * nk);
  acc.knull = (uint8_t *)malloc(acc.alloc_groups * nk);
  acc.st = (ostate *)malloc(sizeof(ostate) * acc.alloc_groups * (na ? na : 1));
  int64_t *pos = (int64_t *)calloc(n_threads, sizeof(int64_t));
  for (int64_t g = 0; g < G; g++) {
    int best = -1;
    for (int t = 0; t < n_threads; t++)
      if (pos[t] < W[t].acc.n_groups && (best < 0 || W[t].first[pos[t]] < W[best].first[pos[best]])) best = t;
    const int64_t s = pos[best]++;
    memcpy(acc.keys + g * nk, W[best].acc.keys + s * nk, sizeof(uint64_t) * nk);
    memcpy(acc.knull + g * nk, W[best].acc.knull + s * nk, nk);
    memcpy(acc.st + g * na, W[best].acc.st + s * na, sizeof(ostate) * na);
  }
  for (int t = 0; t < n_threads; t++) {
    omap_free(&W[t].acc);
    free(W[t].first);
  }
  free(pos);
  *out = finalize(&P, &acc);
  free(acc.keys); free(acc.knull); free(acc.st);
  free(W); free(th);
  plan_free(&P);
  return 0;
}

/* Filter-only: ascending indices of passing rows (scanFilterIndices,
 * src/operators.ts:439-466). */
int oracle_filter_select(int64_t n_rows, int32_t n_cols, const qm_column *cols,
                         const qm_query *q, uint32_t *out, int64_t max_out,
                         int64_t *count) {
  oplan P;
  int rc = plan_build(&P, n_rows, n_cols, cols, q, 0);
  if (rc) { plan_free(&P); return rc; }
  int64_t n = 0;
  for (int64_t r = 0; r < n_rows; r++) {
    if (!row_pass(&P, r)) continue;
    if (n < max_out) out[n] = (uint32_t)r;
    n++;
  }
  *count = n;
  plan_free(&P);
  return n > max_out ? QM_ERR_CAPACITY : 0;
}

int64_t oracle_result_num_rows(const oresult *r) { return r->n_rows; }
int32_t oracle_result_num_columns(const oresult *r) { return r->n_cols; }

int oracle_result_column(const oresult *r, int32_t i, qm_result_col *out) {
  if (i < 0 || i >= r->n_cols) return QM_ERR_INVALID;
  const ocolout *o = &r->cols[i];
  out->name = o->name; out->dtype = o->dtype; out->is_key = o->is_key;
  out->n_rows = r->n_rows; out->data = o->data;
  out->null_bitmap = o->any_null ? o->nulls : NULL;
  return 0;
}

/* Per float SUM cell: 113-bit sum (hi+lo) and sum of |x|; per float AVG
 * cell: the 113-bit mean and the mean of |x|. */
int oracle_result_diag(const oresult *r, int32_t i, const double **xhi,
                       const double **xlo, const double **abssum) {
  if (i < 0 || i >= r->n_cols) return QM_ERR_INVALID;
  *xhi = r->cols[i].xsum_hi; *xlo = r->cols[i].xsum_lo; *abssum = r->cols[i].abssum;
  return 0;
}

void oracle_result_destroy(oresult *r) {
  if (!r) return;
  for (int i = 0; i < r->n_cols; i++) {
    free(r->cols[i].name); free(r->cols[i].data); free(r->cols[i].nulls);
    free(r->cols[i].xsum_hi); free(r->cols[i].xsum_lo); free(r->cols[i].abssum);
  }
  free(r->cols);
  free(r);
}
