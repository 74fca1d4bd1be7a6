"""Pin the CPU oracle to the reference's own known answers (CPU only).

Sources (reference repository paths):
  * src/partial-agg.test.ts:34-178   partial aggregation known answers
  * wasm/src/query/vector_engine.zig:2701-2722   HashGroupBy basic
  * src/operators-conformance.test.ts:98-113, :408-447   5M-row GROUP BY
    conformance; DuckDB is absent here, so the expected values are the
    closed-form sums of the generateRows formula
  * wasm/tests/conformance/fixtures/*.expected.json   filter semantics
    (committed as tests/golden/filter_fixtures.json by
    tests/golden/make_golden.py)
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
from querymode_b200 import datagen
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "filter_fixtures.json")


def col(res, name):
    return res.column(name).pyvalues()


def test_sum_over_rows():
    # partial-agg.test.ts:34-47: sum 60, count 3
    q = QueryDescriptor(aggregates=[AggregateOp("sum", "amount"), AggregateOp("count", "amount")])
    r = oracle.run({"amount": np.array([10.0, 20.0, 30.0])}, q)
    assert col(r, "sum_amount") == [60.0]
    assert col(r, "count_amount") == [3]


def test_group_sum_by_key():
    # partial-agg.test.ts:49-67: us -> 40, eu -> 25 (region as dictionary codes)
    q = QueryDescriptor(group_by=["region"], aggregates=[AggregateOp("sum", "amount")])
    r = oracle.run({"region": np.array([0, 1, 0, 1], np.int32),
                    "amount": np.array([10.0, 20.0, 30.0, 5.0])}, q)
    assert col(r, "region") == [0, 1]  # first-seen order: us, eu
    assert col(r, "sum_amount") == [40.0, 25.0]


def test_merge_two_partials():
    # partial-agg.test.ts:69-89: [10, 20] + [5, 100] -> 135 / 4 / 5 / 100
    q = QueryDescriptor(aggregates=[AggregateOp("sum", "amount"), AggregateOp("count", "amount"),
                                    AggregateOp("min", "amount"), AggregateOp("max", "amount")])
    r = oracle.run({"amount": np.array([10.0, 20.0, 5.0, 100.0])}, q, batch_rows=2)
    assert col(r, "sum_amount") == [135.0]
    assert col(r, "count_amount") == [4]
    assert col(r, "min_amount") == [5.0]
    assert col(r, "max_amount") == [100.0]


def test_finalize_avg_and_friends():
    # partial-agg.test.ts:123-145
    q = QueryDescriptor(aggregates=[AggregateOp("avg", "v"), AggregateOp("sum", "v"), AggregateOp("min", "v"),
                                    AggregateOp("max", "v"), AggregateOp("count", "v")])
    r = oracle.run({"v": np.array([10.0, 20.0, 30.0])}, q)
    assert (col(r, "avg_v"), col(r, "sum_v"), col(r, "min_v"), col(r, "max_v"), col(r, "count_v")) == \
        ([20.0], [60.0], [10.0], [30.0], [3])


def test_nan_inf_group_keys():
    # partial-agg.test.ts:147-178: NaN -> 3, Infinity -> 3, -Infinity -> 4
    q = QueryDescriptor(group_by=["g"], aggregates=[AggregateOp("sum", "v")])
    r = oracle.run({"g": np.array([math.nan, math.nan, math.inf, -math.inf]),
                    "v": np.array([1.0, 2.0, 3.0, 4.0])}, q)
    g = col(r, "g")
    s = col(r, "sum_v")
    assert len(g) == 3
    assert math.isnan(g[0]) and s[0] == 3.0
    assert g[1] == math.inf and s[1] == 3.0
    assert g[2] == -math.inf and s[2] == 4.0


def test_initial_state_semantics():
    # initPartialAggState (src/partial-agg.ts:46-61): min starts at Infinity,
    # max at -Infinity; NaN never wins '<' / '>' but is counted and summed.
    q = QueryDescriptor(aggregates=[AggregateOp("min", "v"), AggregateOp("max", "v"), AggregateOp("sum", "v"),
                                    AggregateOp("count", "v")])
    r = oracle.run({"v": np.array([math.nan])}, q)
    assert col(r, "min_v") == [math.inf]
    assert col(r, "max_v") == [-math.inf]
    assert math.isnan(col(r, "sum_v")[0])
    assert col(r, "count_v") == [1]


def test_empty_ungrouped_row():
    # resolveValue: count 0 -> COUNT 0, others NULL (src/partial-agg.ts:105-111)
    q = QueryDescriptor(filters=[FilterOp("v", "gt", 100)],
                        aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    r = oracle.run({"v": np.array([1.0, 2.0])}, q)
    assert col(r, "sum_v") == [None] and col(r, "count_*") == [0]


def test_hash_group_by_basic():
    # wasm/src/query/vector_engine.zig:2701-2722: 3 groups, key 1 -> sum 90, count 3
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    r = oracle.run({"k": np.array([1, 2, 1, 2, 1, 3], np.int64),
                    "v": np.array([10.0, 20.0, 30.0, 40.0, 50.0, 60.0])}, q)
    assert r.n_rows == 3
    i = col(r, "k").index(1)
    assert col(r, "sum_v")[i] == 90.0 and col(r, "count_*")[i] == 3


def generate_rows_expected(n):
    i = np.arange(n, dtype=np.int64)
    amount = (i * 7 + 13) % 1000
    region = i % 4
    exp = {}
    for r in range(4):
        a = amount[region == r]
        exp[r] = (int(a.sum()), int(a.min()), int(a.max()), int(a.size))
    return exp


def test_generate_rows_5m_by_region():
    # src/operators-conformance.test.ts:408-447 (MockOperator 4096-row batches)
    n = 5_000_000
    cols = datagen.generate_rows(n)
    q = QueryDescriptor(group_by=["region"], aggregates=[
        AggregateOp("sum", "amount", "sum_amount"), AggregateOp("avg", "amount", "avg_amount"),
        AggregateOp("min", "amount", "min_amount"), AggregateOp("max", "amount", "max_amount"),
        AggregateOp("count", "amount", "cnt")])
    r = oracle.run(cols, q, batch_rows=4096)
    exp = generate_rows_expected(n)
    assert col(r, "region") == [0, 1, 2, 3]
    for k, reg in enumerate(col(r, "region")):
        s, mn, mx, c = exp[reg]
        assert col(r, "sum_amount")[k] == float(s)
        assert col(r, "min_amount")[k] == mn
        assert col(r, "max_amount")[k] == mx
        assert col(r, "cnt")[k] == c
        assert abs(col(r, "avg_amount")[k] - s / c) < 1e-5  # toBeCloseTo(..., 5)


def load_golden():
    with open(GOLDEN) as f:
        return json.load(f)


def golden_columns(g):
    cols = {}
    np_types = {"int64": np.int64, "int32": np.int32, "float64": np.float64}
    for name, vals in g["table"].items():
        nulls = np.array([v is None for v in vals])
        arr = np.array([0 if v is None else v for v in vals], dtype=np_types[g["dtypes"][name]])
        cols[name] = Column(arr, nulls)
    return cols


def golden_query(case):
    def f(d):
        v = d.get("value")
        if isinstance(v, list):
            v = [float(x) if isinstance(x, float) else x for x in v]
        return FilterOp(d["column"], d["op"], v)
    return QueryDescriptor(filters=[f(x) for x in case["filters"]],
                           filter_groups=[[f(x) for x in grp] for grp in case["filter_groups"]]
                           if case["filter_groups"] else None)


@pytest.mark.parametrize("case", load_golden()["cases"], ids=lambda c: c["name"])
def test_filter_fixtures(case):
    g = load_golden()
    got = oracle.filter_select(golden_columns(g), golden_query(case))
    assert got.tolist() == case["expected_rows"], case["query"]
