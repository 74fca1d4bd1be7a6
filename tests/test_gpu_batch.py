"""Batched launch (qm_batch_*): every query's result equals the oracle's,
on the first (graph-capturing) run, on a replay, and after retuning."""
import numpy as np
import pytest

import oracle
from querymode_b200 import datagen
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def mixed_batch(seed=5, n=40):
    specs = datagen.batch_specs(n, seed=seed, rows_lo=1e3, rows_hi=3e5, card_lo=1, card_hi=5e4)
    tables = [datagen.batch_table(s) for s in specs]
    queries = [datagen.batch_query(s) for s in specs]
    rng = np.random.default_rng(seed)
    # other shapes: ungrouped, two packed keys, NULLs, int sums
    m = 50_000
    extra = {"a": Column(rng.integers(0, 7, m).astype(np.int32), rng.random(m) < 0.1),
             "b": rng.integers(-3, 3, m).astype(np.int32), "x": Column(rng.normal(size=m), rng.random(m) < 0.2),
             "i": rng.integers(-2**40, 2**40, m).astype(np.int64)}
    tables += [extra, extra, extra]
    queries += [QueryDescriptor(filters=[FilterOp("b", "gte", 0)],
                                aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "*"), AggregateOp("max", "i")]),
                QueryDescriptor(group_by=["a", "b"], aggregates=[AggregateOp("sum", "i"), AggregateOp("avg", "x"),
                                                                  AggregateOp("count", "x")]),
                QueryDescriptor(filters=[FilterOp("x", "gt", 5.0)], group_by=["a"],
                                aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "*")])]
    return tables, queries


def test_batch_matches_oracle(ctx):
    tables, queries = mixed_batch()
    handles = [ctx.table(t) for t in tables]
    refs = [oracle.run(t, q) for t, q in zip(tables, queries)]
    b = ctx.batch(handles, queries)
    try:
        for run in range(2):  # capture, then replay
            res = b.run()
            for i, (g, r) in enumerate(zip(res, refs)):
                assert_same(g, r, ctx_msg=f"run {run} query {i}")
        # the persistent kernel, default and retuned
        b.set_mode(0)
        for tuning in ({}, {"chunk_tiles": 64, "local_kb": 0, "blocks_per_sm": 1}):
            b.set_tuning(**tuning)
            res = b.run()
            for i, (g, r) in enumerate(zip(res, refs)):
                assert_same(g, r, ctx_msg=f"persistent {tuning} query {i}")
        st = b.stats()
        assert st["rows"] == sum(len(next(iter(t.values())).values if hasattr(next(iter(t.values())), "values")
                                     else next(iter(t.values()))) for t in tables)
    finally:
        b.close()


def test_batch_equals_single_queries(ctx):
    specs = datagen.batch_specs(16, seed=9, rows_lo=1e4, rows_hi=2e6, card_lo=4, card_hi=2e5)
    tables = [ctx.table(datagen.batch_table(s)) for s in specs]
    queries = [datagen.batch_query(s) for s in specs]
    singles = [t.run(q) for t, q in zip(tables, queries)]
    b = ctx.batch(tables, queries)
    try:
        for g, r in zip(b.run(), singles):
            assert_same(g, r)
    finally:
        b.close()


def test_batch_dense_keys_beyond_shared_memory(ctx):
    # dense int32 keys whose direct tables exceed shared memory (block-local
    # hash, then the global table) beside ones that fit, NULL keys included
    rng = np.random.default_rng(13)
    tables, queries = [], []
    for card, n in ((9_000, 1_500_000), (20_000, 2_000_000), (300, 400_000), (4_000, 600_000)):
        cols = {"key": Column(rng.integers(0, card, n).astype(np.int32), rng.random(n) < 0.001),
                "f": rng.integers(0, 10_000, n).astype(np.int32), "v": rng.lognormal(size=n)}
        tables.append(cols)
        queries.append(QueryDescriptor(filters=[FilterOp("f", "lt", 7000)], group_by=["key"],
                                       aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*"),
                                                   AggregateOp("min", "v"), AggregateOp("max", "v")]))
    handles = [ctx.table(t) for t in tables]
    refs = [oracle.run(t, q) for t, q in zip(tables, queries)]
    b = ctx.batch(handles, queries)
    try:
        for run in range(2):
            for i, (g, r) in enumerate(zip(b.run(), refs)):
                assert_same(g, r, ctx_msg=f"run {run} query {i}")
    finally:
        b.close()


def test_batch_overflow_reruns_alone(ctx):
    # a batch planned on borrowed device columns whose keys are then rewritten
    # to far more distinct values than the cached estimate: the query's
    # batched table overflows, and it is run again alone (where its table
    # regrows) to the oracle's answer
    import torch
    rng = np.random.default_rng(17)
    n = 300_000
    k0 = rng.integers(-(1 << 62), 1 << 62, 50).astype(np.int64)[rng.integers(0, 50, n)]
    v = rng.normal(size=n)
    dk = torch.from_numpy(k0).cuda()
    t = ctx.table({"key": dk, "v": torch.from_numpy(v).cuda()})
    q = QueryDescriptor(group_by=["key"], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    other = {"key": rng.integers(0, 7, 1000).astype(np.int32), "v": rng.normal(size=1000)}
    t2 = ctx.table(other)
    b = ctx.batch([t, t2], [q, q])
    try:
        for g, r in zip(b.run(), [oracle.run({"key": k0, "v": v}, q), oracle.run(other, q)]):
            assert_same(g, r)
        k1 = rng.integers(-(1 << 62), 1 << 62, 5000).astype(np.int64)[rng.integers(0, 5000, n)]
        dk.copy_(torch.from_numpy(k1))
        res = b.run()
        assert res[0].stats.retries >= 1, res[0].stats  # run alone, regrown
        assert_same(res[0], oracle.run({"key": k1, "v": v}, q))
        assert_same(res[1], oracle.run(other, q))
    finally:
        b.close()
        t.close()
        t2.close()


@pytest.mark.parametrize("mode", [1, 0])
def test_batch_waves_keep_results(ctx, mode):
    """The batch cut into 1, 3 or 8 waves (each wave's results copied back
    while later waves run), per-query launches and the persistent kernel:
    every query still equals the oracle, on capture and on replay."""
    tables, queries = mixed_batch(seed=21, n=30)
    handles = [ctx.table(t) for t in tables]
    refs = [oracle.run(t, q) for t, q in zip(tables, queries)]
    b = ctx.batch(handles, queries)
    try:
        b.set_mode(mode)
        for waves in (3, 8, 1, 0):
            b.set_waves(waves)
            for run in range(2):
                for i, (g, r) in enumerate(zip(b.run(), refs)):
                    assert_same(g, r, ctx_msg=f"mode {mode} waves {waves} run {run} query {i}")
    finally:
        b.close()
