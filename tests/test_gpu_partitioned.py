"""Partitioned aggregation (strategy 3, opt-in with qm_tuning.partitioned):
group tables larger than a block's shared memory with many selected rows per
group are aggregated partition by partition in shared memory.  Each shape below takes that route (checked on
the result's strategy) and must equal the oracle: keys and first-seen order,
COUNT, integer SUM / MIN / MAX and float MIN / MAX bit-exact, float SUM /
AVG within 1e-12 (tests/helpers.py)."""
import numpy as np
import pytest

import oracle
from querymode_b200 import datagen
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu

AGGS = [AggregateOp("sum", "v"), AggregateOp("min", "v"), AggregateOp("max", "v"), AggregateOp("count", "*"),
        AggregateOp("avg", "v"), AggregateOp("sum", "w"), AggregateOp("count", "v"), AggregateOp("max", "w")]


def columns(rng, n, key):
    v = rng.normal(size=n) * 100
    v[rng.random(n) < 0.001] = -0.0
    return {"key": key, "v": Column(v, rng.random(n) < 0.02), "w": rng.integers(-1000, 1000, n).astype(np.int32),
            "f": rng.integers(0, 100, n).astype(np.int32)}


@pytest.fixture(autouse=True)
def partitioned(ctx):
    ctx.set_tuning(partitioned=1)
    try:
        yield
    finally:
        ctx.set_tuning()


def check(ctx, cols, q, strategy=3):
    g = ctx.table(cols).run(q)
    assert g.stats.strategy == strategy, g.stats
    assert_same(g, oracle.run_full(cols, q))


def test_direct_keys_no_filter(ctx):
    rng = np.random.default_rng(1)
    n = 8_000_000
    check(ctx, columns(rng, n, rng.integers(0, 40_000, n).astype(np.int32)),
          QueryDescriptor(group_by=["key"], aggregates=AGGS))


def test_direct_keys_filtered_with_null_keys(ctx):
    rng = np.random.default_rng(2)
    n = 6_000_000
    key = Column(rng.integers(-5_000, 25_000, n).astype(np.int64), rng.random(n) < 0.01)
    check(ctx, columns(rng, n, key), QueryDescriptor(filters=[FilterOp("f", "lt", 70)], group_by=["key"],
                                                     aggregates=AGGS))


def test_hashed_keys(ctx):
    rng = np.random.default_rng(3)
    n = 8_000_000
    universe = rng.integers(-(1 << 62), 1 << 62, 60_000).astype(np.int64)
    universe[7] = np.iinfo(np.int64).min  # the empty-slot sentinel as a real key
    key = universe[rng.integers(0, len(universe), n)]
    check(ctx, columns(rng, n, key), QueryDescriptor(filters=[FilterOp("f", "gte", 30)], group_by=["key"],
                                                     aggregates=AGGS))


def test_two_column_keys(ctx):
    rng = np.random.default_rng(4)
    n = 6_000_000
    cols = columns(rng, n, rng.integers(0, 300, n).astype(np.int32))
    cols["k2"] = rng.integers(0, 200, n).astype(np.int64)
    check(ctx, cols, QueryDescriptor(group_by=["key", "k2"], aggregates=AGGS))


def test_wide_keys_unfiltered(ctx):
    """wide_keys 50M rows over 2^18 keys, unfiltered (128 partitions of the
    direct table)."""
    cols = datagen.wide_keys(50_000_000, seed=9, n_keys=1 << 18)
    check(ctx, cols, datagen.wide_keys_query(False))


def test_too_many_partitions_keeps_the_scan(ctx):
    """A direct table of more windows than the partition cap (the 2^22-key
    shape) keeps the scan and its key-range passes."""
    cols = datagen.wide_keys(20_000_000, seed=10, n_keys=1 << 22)
    q = datagen.wide_keys_query(False)
    g = ctx.table(cols).run(q)
    assert g.stats.strategy != 3
    assert_same(g, oracle.run_full(cols, q))


def test_selective_filter_keeps_the_scan(ctx):
    """A selective filter (below a quarter of the rows) keeps the fused scan."""
    rng = np.random.default_rng(5)
    n = 6_000_000
    cols = columns(rng, n, rng.integers(0, 40_000, n).astype(np.int32))
    g = ctx.table(cols).run(QueryDescriptor(filters=[FilterOp("f", "lt", 10)], group_by=["key"], aggregates=AGGS))
    assert g.stats.strategy != 3


def test_off_by_default(ctx):
    ctx.set_tuning()
    rng = np.random.default_rng(6)
    n = 6_000_000
    cols = columns(rng, n, rng.integers(0, 40_000, n).astype(np.int32))
    g = ctx.table(cols).run(QueryDescriptor(group_by=["key"], aggregates=AGGS))
    assert g.stats.strategy != 3
