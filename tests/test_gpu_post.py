"""Post-aggregate ORDER BY / LIMIT / OFFSET on the GPU result against the
reference's TopKOperator / InMemorySortOperator / LimitOperator restated
(oracle/post.py) over the oracle's result: same rows in the same order,
ties included."""
import dataclasses

import numpy as np
import pytest

import oracle
from oracle.post import post_aggregate
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def table(seed=2, n=400_000):
    rng = np.random.default_rng(seed)
    key = (rng.zipf(1.3, n) % 3000).astype(np.int64)
    x = rng.normal(size=n) * 100
    x[rng.random(n) < 0.01] = np.nan
    return {"key": Column(key, rng.random(n) < 0.002),
            "qty": rng.integers(1, 100, n).astype(np.int32),
            "price": Column(np.round(rng.random(n) * 1000, 1), rng.random(n) < 0.05),
            "big": rng.integers(-2**62, 2**62, n).astype(np.int64),
            "x": x}


BASE = QueryDescriptor(filters=[FilterOp("qty", "gt", 5)], group_by=["key"],
                       aggregates=[AggregateOp("count", "*", "n"), AggregateOp("sum", "qty", "sq"),
                                   AggregateOp("min", "price", "lo"), AggregateOp("max", "price", "hi"),
                                   AggregateOp("sum", "big", "sb"), AggregateOp("min", "x", "mx")])

CASES = [
    dict(sort_column="n", sort_desc=True, limit=10),
    dict(sort_column="n", sort_desc=False, limit=50, offset=5),
    dict(sort_column="lo", sort_desc=False),
    dict(sort_column="hi", sort_desc=True, offset=100),
    dict(sort_column="key", sort_desc=True, limit=20),
    dict(sort_column="sq", sort_desc=True, limit=7),
    dict(sort_column="sb", sort_desc=True, limit=5),
    dict(sort_column="sb", sort_desc=False),
    dict(sort_column="mx", sort_desc=False, limit=30),
    dict(limit=10, offset=3),
    dict(offset=2990),
    dict(sort_column="nope", limit=5),
    dict(sort_column="n", sort_desc=True, limit=100_000),
    dict(sort_column="n", limit=0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: ",".join(f"{k}={v}" for k, v in c.items()))
def test_order_limit_matches_reference_operators(ctx, case):
    cols = table()
    ref = oracle.run(cols, BASE)
    want = post_aggregate(ref, case.get("sort_column"), case.get("sort_desc", False), case.get("limit"),
                          case.get("offset", 0))
    q = dataclasses.replace(BASE, **case)
    got = ctx.table(cols).run(q)
    assert got.n_rows == want.n_rows
    assert_same(got, want, ctx_msg=str(case))
    # the same through a streamed aggregation
    s = ctx.aggregate(q)
    s.push(cols)
    assert_same(s.finish(), want, ctx_msg=f"stream {case}")


def test_topk_over_many_groups_with_ties(ctx):
    rng = np.random.default_rng(8)
    n = 2_000_000
    cols = {"k": rng.integers(0, 200_000, n).astype(np.int64), "v": rng.integers(0, 3, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("count", "*", "n"), AggregateOp("max", "v", "m")])
    ref = oracle.run(cols, q, threads=8)
    for sc, desc, lim, off in (("n", True, 1000, 0), ("m", False, 5000, 17), ("n", False, None, 0)):
        want = post_aggregate(ref, sc, desc, lim, off)
        got = ctx.table(cols).run(dataclasses.replace(q, sort_column=sc, sort_desc=desc, limit=lim, offset=off))
        assert_same(got, want, ctx_msg=f"{sc} {desc} {lim} {off}")
