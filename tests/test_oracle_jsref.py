"""Pin the C oracle against the literal restatement (oracle/jsref.py), which
keeps the reference's string group keys and Map order, on seeded random
tables with NULLs, NaN, +-0, +-Infinity, large int64 values, JS number /
bigint thresholds of every op, OR groups and several batch sizes (CPU only).
"""
import math

import numpy as np
import pytest

import oracle
from oracle import jsref
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, BigInt, FilterOp, QueryDescriptor

N = 300


def make_table(rng, n=N):
    i32 = rng.integers(-5, 6, n).astype(np.int32)
    i64 = rng.choice(np.array([-(2**62), -7, -1, 0, 1, 3, 7, 2**53 + 1, 2**62], np.int64), n)
    f64 = rng.choice(np.array([-2.5, -0.0, 0.0, 0.5, 1.0, 3.25, math.nan, math.inf, -math.inf, 1e300]), n)
    f32 = rng.choice(np.array([-1.5, 0.0, 2.25, 7.0], np.float32), n)
    g32 = rng.integers(0, 4, n).astype(np.int32)
    cols = {
        "i32": Column(i32, rng.random(n) < 0.1),
        "i64": Column(i64, rng.random(n) < 0.1),
        "f64": Column(f64, rng.random(n) < 0.1),
        "f32": Column(f32, None),
        "g32": Column(g32, None),
        "gf": Column(rng.choice(np.array([-0.0, 0.0, math.nan, 1.5]), n), rng.random(n) < 0.05),
    }
    return cols


def to_js(cols):
    out = {}
    for name, c in cols.items():
        vals = []
        for k, v in enumerate(c.values):
            if c.nulls is not None and c.nulls[k]:
                vals.append(None)
            elif c.values.dtype == np.int64:
                vals.append(int(v))
            else:
                vals.append(float(v))
        out[name] = vals
    return out


THRESH = [0, 1, -1, 2.5, -2.5, 0.5, 7, math.nan, math.inf, -math.inf, 2**53 + 1.0, 1e300]
BIGS = [BigInt(0), BigInt(3), BigInt(-7), BigInt(2**53 + 1)]
OPS = ["eq", "neq", "lt", "lte", "gt", "gte", "between", "not_between", "is_null", "is_not_null"]


def rand_filter(rng):
    col = str(rng.choice(["i32", "i64", "f64", "f32"]))
    op = str(rng.choice(OPS))

    def val():
        if rng.random() < 0.2 and not (col in ("f64", "f32") and op in ("between", "not_between")):
            return BIGS[rng.integers(len(BIGS))]
        return THRESH[rng.integers(len(THRESH))]
    if op in ("between", "not_between"):
        v = [val(), val()]
        if col in ("f64", "f32"):
            v = [float(x) for x in v]
        return FilterOp(col, op, v)
    if op in ("is_null", "is_not_null"):
        return FilterOp(col, op)
    return FilterOp(col, op, val())


def rand_query(rng, stream_keys=False):
    """stream_keys: only key shapes a stream of batches can group by (no
    table statistics to pack several columns into one word)."""
    filters = [rand_filter(rng) for _ in range(rng.integers(0, 3))]
    groups = None
    if rng.random() < 0.3:
        groups = [[rand_filter(rng) for _ in range(rng.integers(1, 3))] for _ in range(rng.integers(1, 3))]
    gb = [["g32"], ["i64"], ["gf"], ["i32"], [], ["g32", "i32"], ["i32", "g32"]][rng.integers(7)]
    if stream_keys and len(gb) > 1:
        gb = ["g32"]
    aggs = [AggregateOp("count", "*")]
    for _ in range(rng.integers(1, 5)):
        aggs.append(AggregateOp(str(rng.choice(["sum", "avg", "min", "max", "count"])),
                                str(rng.choice(["i32", "i64", "f64", "f32"]))))
    # unique aliases
    seen, out = set(), []
    for a in aggs:
        if a.out_name not in seen:
            seen.add(a.out_name)
            out.append(a)
    return QueryDescriptor(filters=filters, filter_groups=groups, group_by=gb, aggregates=out)


def same_value(a, b):
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, float) and math.isnan(a) or isinstance(b, float) and math.isnan(b):
        return isinstance(a, float) and isinstance(b, float) and math.isnan(a) and math.isnan(b)
    if a == 0 and b == 0 and isinstance(a, float) and isinstance(b, float):
        return math.copysign(1, a) == math.copysign(1, b)
    return a == b


@pytest.mark.parametrize("seed", range(60))
def test_oracle_matches_literal_js(seed):
    rng = np.random.default_rng(1000 + seed)
    cols = make_table(rng)
    q = rand_query(rng)
    batch = int(rng.choice([0, 7, 64, 1000]))
    js_rows = jsref.run(to_js(cols), q, batch)
    r = oracle.run(cols, q, batch_rows=batch)
    from querymode_b200.rows import result_to_rows
    c_rows = result_to_rows(r, bool(q.group_by))
    assert len(c_rows) == len(js_rows), (q, len(c_rows), len(js_rows))
    for a, b in zip(c_rows, js_rows):
        assert list(a.keys()) == list(b.keys())
        for k in a:
            assert same_value(a[k], b[k]), (seed, k, a[k], b[k], q)


@pytest.mark.parametrize("seed", range(40))
def test_filter_select_matches_literal_js(seed):
    rng = np.random.default_rng(5000 + seed)
    cols = make_table(rng)
    q = rand_query(rng)
    js = to_js(cols)
    rows = [{c: js[c][r] for c in js} for r in range(N)]
    exp = [r for r in range(N) if jsref.row_passes_filters(rows[r], q.filters, q.filter_groups)]
    got = oracle.filter_select(cols, q)
    assert got.tolist() == exp, q


def test_js_number_strings():
    cases = {1.0: "1", 1.5: "1.5", 1e21: "1e+21", 1e20: "100000000000000000000", 1e-7: "1e-7",
             0.000001: "0.000001", 123456789012345680000.0: "123456789012345680000", -0.0: "0",
             2.0 ** 60: "1152921504606847000", 0.1: "0.1", 5e-324: "5e-324"}
    for x, s in cases.items():
        assert jsref.js_num_str(x) == s, (x, jsref.js_num_str(x), s)
    # key restoration: int64 keys beyond 2^53 that do not round-trip stay bigint
    assert jsref.restore_key_part("9007199254740993") == 9007199254740993
    assert isinstance(jsref.restore_key_part("9007199254740993"), int)
    assert isinstance(jsref.restore_key_part("5"), float)
