"""Large results against the oracle — direct-indexed ones emitted in output
order (the first-row bitmap walk used for resident tables of at least 2^20
group slots), hashed ones at their ranks: keys and first-seen order, COUNT,
integer SUM and float MIN / MAX bit-exact, float SUM / AVG within the path's
tolerance (tests/helpers.py).
Covers NULL keys (the direct table's NULL slot), digit-packed two-column keys
with a nullable column, a filter that leaves most slots empty, and a
post-aggregate ORDER BY / LIMIT over the walked result (finalizePartialAgg,
src/partial-agg.ts:306-352; first-seen group order, src/types.ts:10-18)."""
import numpy as np
import pytest

import dataclasses

import oracle
from oracle.post import post_aggregate
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu

AGGS = [AggregateOp("sum", "v"), AggregateOp("count", "*"), AggregateOp("min", "v"), AggregateOp("max", "w"),
        AggregateOp("avg", "v"), AggregateOp("sum", "w")]


def run(ctx, cols, q):
    t = ctx.table(cols)
    g = t.run(q)
    t.close()
    return g


def test_int64_keys_with_nulls(ctx):
    rng = np.random.default_rng(11)
    n = 6_000_000
    key = Column(rng.integers(-1000, (1 << 21) - 1000, n).astype(np.int64), rng.random(n) < 0.05)
    cols = {"key": key, "v": rng.normal(size=n) * 10, "w": rng.integers(-50, 50, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["key"], aggregates=AGGS)
    g = run(ctx, cols, q)
    assert g.n_rows > 1_500_000
    assert_same(g, oracle.run_full(cols, q), ctx_msg="int64 keys with NULLs")


def test_two_packed_keys_nullable(ctx):
    rng = np.random.default_rng(12)
    n = 5_000_000
    cols = {"a": rng.integers(0, 1500, n).astype(np.int32),
            "b": Column(rng.integers(0, 1000, n).astype(np.int64), rng.random(n) < 0.02),
            "v": rng.random(n), "w": rng.integers(0, 7, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["a", "b"], aggregates=AGGS)
    g = run(ctx, cols, q)
    assert g.n_rows > 1_000_000
    assert_same(g, oracle.run_full(cols, q), ctx_msg="packed keys")


def test_filtered_sparse_slots(ctx):
    rng = np.random.default_rng(13)
    n = 8_000_000
    cols = {"key": rng.integers(0, 1 << 22, n).astype(np.int32), "f": rng.integers(0, 100, n).astype(np.int32),
            "v": rng.normal(size=n), "w": rng.integers(-9, 9, n).astype(np.int32)}
    q = QueryDescriptor(filters=[FilterOp("f", "lt", 60)], group_by=["key"], aggregates=AGGS)
    assert_same(run(ctx, cols, q), oracle.run_full(cols, q), ctx_msg="filtered")


def test_order_by_limit_after_walk(ctx):
    rng = np.random.default_rng(14)
    n = 4_000_000
    cols = {"key": rng.integers(0, 1 << 21, n).astype(np.int64), "v": rng.normal(size=n),
            "w": rng.integers(0, 1000, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["key"], aggregates=AGGS)
    want = post_aggregate(oracle.run_full(cols, q), "sum_w", True, 1000, 0)
    got = run(ctx, cols, dataclasses.replace(q, sort_column="sum_w", sort_desc=True, limit=1000))
    assert_same(got, want, ctx_msg="order by / limit")


def test_hashed_keys_with_sentinel_and_nulls(ctx):
    """A hash table of over 2^20 slots (800K distinct random int64 keys), the
    empty-slot sentinel as a real key and NULL keys (the slot-order emit of
    large hashed results, beside the walk of the direct ones)."""
    rng = np.random.default_rng(15)
    n = 5_000_000
    universe = rng.integers(-(1 << 62), 1 << 62, 800_000).astype(np.int64)
    universe[5] = np.iinfo(np.int64).min
    key = Column(universe[rng.integers(0, len(universe), n)], rng.random(n) < 0.01)
    cols = {"key": key, "v": rng.normal(size=n), "w": rng.integers(-3, 3, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["key"], aggregates=AGGS)
    g = run(ctx, cols, q)
    assert g.n_rows > 700_000
    assert_same(g, oracle.run_full(cols, q), ctx_msg="hashed keys")


def test_chunked_dense_result_with_null_outputs(ctx):
    """A dense direct table of 2^22 + 1 slots (4M groups of 12M rows): the
    result is laid out before its group count is known and emitted and copied
    in row chunks.  30 % NULL values leave some groups with NULL SUM / MIN /
    AVG (the chunks' NULL-bitmap words), and 1 % NULL keys the NULL group."""
    rng = np.random.default_rng(16)
    n = 12_000_000
    key = Column(rng.integers(0, 1 << 22, n).astype(np.int64), rng.random(n) < 0.01)
    cols = {"key": key, "v": Column(rng.normal(size=n), rng.random(n) < 0.3),
            "w": rng.integers(-100, 100, n).astype(np.int32)}
    q = QueryDescriptor(group_by=["key"], aggregates=AGGS)
    g = run(ctx, cols, q)
    assert g.n_rows > 3_900_000
    assert g.column("sum_v").nulls is not None and g.column("sum_v").nulls.any()
    assert_same(g, oracle.run_full(cols, q), ctx_msg="chunked dense result")
