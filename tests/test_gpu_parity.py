"""GPU path vs the CPU oracle, through the C ABI (libqm_gpu.so via ctypes).

Bit-exact: group keys and their first-seen order, COUNT, integer SUM / MIN /
MAX, float MIN / MAX (the sign of a zero included).  Float SUM / AVG: within
1e-12 relative (tests/helpers.py states the fallback for cancelling sums).
"""
import math

import numpy as np
import pytest

import oracle
from querymode_b200 import _abi as A
from querymode_b200 import datagen
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, BigInt, FilterOp, QueryDescriptor
from tests.helpers import assert_same
from tests.test_oracle_golden import golden_columns, golden_query, load_golden
from tests.test_oracle_jsref import make_table, rand_query

pytestmark = pytest.mark.gpu


def run_both(ctx, cols, q, batch_rows=0):
    t = ctx.table(cols)
    g = t.run(q)
    r = oracle.run(cols, q, batch_rows=batch_rows)
    return g, r


def test_orders_1m(ctx):
    cols = datagen.orders()
    g, r = run_both(ctx, cols, datagen.orders_query())
    assert g.n_rows == 16
    assert_same(g, r)
    assert g.stats.rows_selected == int((cols["status"] == 1).sum())


def test_events_4m(ctx):
    cols = datagen.events(4_000_000, seed=11)
    q = datagen.events_query()
    g, r = run_both(ctx, cols, q)
    assert g.n_rows > 1000
    assert_same(g, r)


def test_wide_keys_filtered_and_full(ctx):
    cols = datagen.wide_keys(6_000_000, seed=12, n_keys=1 << 20)
    for filtered in (True, False):
        g, r = run_both(ctx, cols, datagen.wide_keys_query(filtered))
        assert_same(g, r, ctx_msg=f"filtered={filtered}")


def test_generate_rows_conformance(ctx):
    cols = datagen.generate_rows(5_000_000)
    q = QueryDescriptor(group_by=["region"], aggregates=[
        AggregateOp("sum", "amount", "sum_amount"), AggregateOp("avg", "amount", "avg_amount"),
        AggregateOp("min", "amount", "min_amount"), AggregateOp("max", "amount", "max_amount"),
        AggregateOp("count", "amount", "cnt")])
    g, r = run_both(ctx, cols, q, batch_rows=4096)
    assert_same(g, r)


@pytest.mark.parametrize("seed", range(40))
def test_random_queries(ctx, seed):
    rng = np.random.default_rng(1000 + seed)
    cols = make_table(rng, n=int(rng.choice([300, 5000, 70000])))
    q = rand_query(rng)
    g, r = run_both(ctx, cols, q)
    assert_same(g, r, ctx_msg=str(q))


@pytest.mark.parametrize("seed", range(12))
def test_streamed_batches_and_selection(ctx, seed):
    rng = np.random.default_rng(7000 + seed)
    n = 20000
    cols = make_table(rng, n=n)
    q = rand_query(rng, stream_keys=True)
    batch = int(rng.choice([1000, 4096, 7777]))
    # reference: AggregateOperator over batches whose selection vectors keep
    # every third row (a scan that already filtered)
    keep = np.arange(n) % 3 != 1
    ref_cols = {k: Column(v.values[keep], None if v.nulls is None else v.nulls[keep]) for k, v in cols.items()}
    s = ctx.aggregate(q)
    for b0 in range(0, n, batch):
        b1 = min(n, b0 + batch)
        part = {k: Column(v.values[b0:b1], None if v.nulls is None else v.nulls[b0:b1]) for k, v in cols.items()}
        sel = np.nonzero(keep[b0:b1])[0].astype(np.uint32)
        s.push(part, selection=sel)
    g = s.finish()
    s.close()
    r = oracle.run(ref_cols, q, batch_rows=0)
    assert_same(g, r, ctx_msg=str(q))


@pytest.mark.parametrize("seed", range(20))
def test_filter_select_random(ctx, seed):
    rng = np.random.default_rng(5000 + seed)
    cols = make_table(rng, n=int(rng.choice([300, 10000, 100000])))
    q = rand_query(rng)
    assert ctx.filter_select(cols, q).tolist() == oracle.filter_select(cols, q).tolist()


@pytest.mark.parametrize("case", load_golden()["cases"], ids=lambda c: c["name"])
def test_filter_fixtures_gpu(ctx, case):
    g = load_golden()
    got = ctx.filter_select(golden_columns(g), golden_query(case))
    assert got.tolist() == case["expected_rows"], case["query"]


def test_empty_and_all_filtered(ctx):
    cols = {"k": np.array([1, 2, 3], np.int64), "v": np.array([1.0, 2.0, 3.0])}
    q = QueryDescriptor(filters=[FilterOp("v", "gt", 10)], group_by=["k"],
                        aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    g, r = run_both(ctx, cols, q)
    assert g.n_rows == 0 and r.n_rows == 0
    q2 = QueryDescriptor(filters=[FilterOp("v", "gt", 10)],
                         aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    g, r = run_both(ctx, cols, q2)
    assert g.n_rows == 1 and g.column("count_*").pyvalues() == [0] and g.column("sum_v").pyvalues() == [None]
    assert_same(g, r)
    empty = {"k": np.zeros(0, np.int64), "v": np.zeros(0)}
    g, r = run_both(ctx, empty, q)
    assert g.n_rows == 0 and r.n_rows == 0


def test_extreme_int64_keys_and_sums(ctx):
    imin, imax = np.iinfo(np.int64).min, np.iinfo(np.int64).max
    keys = np.array([imin, imax, 0, imin, -1, imax, imin] * 1000, np.int64)
    vals = np.array([imax, imax, imin, imin, 5, imax, -3] * 1000, np.int64)
    cols = {"k": keys, "v": vals}
    q = QueryDescriptor(group_by=["k"], aggregates=[
        AggregateOp("sum", "v"), AggregateOp("avg", "v"), AggregateOp("min", "v"), AggregateOp("max", "v"),
        AggregateOp("count", "*")])
    g, r = run_both(ctx, cols, q)
    assert_same(g, r)
    sums = g.column("sum_v").pyvalues()
    assert max(abs(s) for s in sums) > 2**63  # beyond int64: exact 128-bit


def test_random_int64_keys_hash_mode(ctx):
    rng = np.random.default_rng(3)
    universe = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, 300_000, dtype=np.int64)
    keys = universe[rng.integers(0, universe.size, 3_000_000)]
    cols = {"k": keys, "v": rng.normal(0, 1, keys.size), "w": rng.integers(-100, 100, keys.size).astype(np.int32)}
    q = QueryDescriptor(filters=[FilterOp("w", "gte", -50)], group_by=["k"],
                        aggregates=[AggregateOp("sum", "v"), AggregateOp("min", "w"), AggregateOp("max", "v"),
                                    AggregateOp("count", "*"), AggregateOp("avg", "w")])
    g, r = run_both(ctx, cols, q)
    assert g.stats.strategy in (1, 2)
    assert_same(g, r)


def test_signed_zero_first_seen_min_max(ctx):
    # strict '<' / '>' keep the first of -0 and 0 (src/partial-agg.ts:80-81)
    v = np.array([0.0, -0.0, 0.0, 5.0, -0.0, 0.0, -0.0, 0.0], np.float64)
    k = np.array([0, 0, 1, 1, 2, 2, 3, 3], np.int32)
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("min", "v"), AggregateOp("max", "v"),
                                                    AggregateOp("sum", "v")])
    big_v = np.tile(v, 5000)
    big_k = np.tile(k, 5000) + np.repeat(np.arange(5000, dtype=np.int32) * 4, 8)
    for cols in ({"k": k, "v": v}, {"k": big_k, "v": big_v}):
        g, r = run_both(ctx, cols, q)
        assert_same(g, r)
    mins = g.column("min_v").values
    assert np.signbit(mins[0]) == False and np.signbit(mins[3]) == True  # noqa: E712


def test_nan_inf_values_and_keys(ctx):
    v = np.array([math.nan, 1.0, math.inf, -math.inf, 2.0, math.nan, math.inf, 3.0])
    k = np.array([math.nan, math.nan, 0.0, -0.0, math.inf, 1.0, 1.0, -math.inf])
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("min", "v"),
                                                    AggregateOp("max", "v"), AggregateOp("avg", "v"),
                                                    AggregateOp("count", "v")])
    g, r = run_both(ctx, {"k": k, "v": v}, q)
    assert_same(g, r)


def test_nullable_keys_and_values(ctx):
    rng = np.random.default_rng(9)
    n = 200_000
    cols = {"k": Column(rng.integers(0, 50, n).astype(np.int64), rng.random(n) < 0.05),
            "x": Column(rng.normal(size=n), rng.random(n) < 0.2),
            "y": Column(rng.integers(-9, 9, n).astype(np.int32), rng.random(n) < 0.3)}
    q = QueryDescriptor(filters=[FilterOp("y", "is_not_null")], group_by=["k"],
                        aggregates=[AggregateOp("count", "x"), AggregateOp("sum", "x"), AggregateOp("min", "y"),
                                    AggregateOp("avg", "y"), AggregateOp("count", "*")])
    g, r = run_both(ctx, cols, q)
    assert_same(g, r)


def test_two_int32_keys_and_f32(ctx):
    rng = np.random.default_rng(4)
    n = 300_000
    cols = {"a": rng.integers(-3, 3, n).astype(np.int32), "b": rng.integers(0, 1000, n).astype(np.int32),
            "f": rng.normal(size=n).astype(np.float32)}
    q = QueryDescriptor(filters=[FilterOp("f", "lt", 0.5)], group_by=["a", "b"],
                        aggregates=[AggregateOp("sum", "f"), AggregateOp("max", "f"), AggregateOp("count", "*")])
    g, r = run_both(ctx, cols, q)
    assert_same(g, r)


def test_wasm_scan_semantics(ctx):
    rng = np.random.default_rng(5)
    n = 50_000
    cols = {"i": Column(rng.integers(-10, 10, n).astype(np.int32), rng.random(n) < 0.1),
            "f": Column(rng.normal(size=n), rng.random(n) < 0.1),
            "k": rng.integers(0, 7, n).astype(np.int32)}
    for flt in ([FilterOp("i", "lt", 2.5)], [FilterOp("f", "eq", 0)], [FilterOp("i", "between", [-0.5, 3.7])],
                [FilterOp("i", "gt", 3e9)], [FilterOp("f", "not_between", [-0.1, 0.1])]):
        q = QueryDescriptor(filters=flt, group_by=["k"], aggregates=[AggregateOp("count", "*")],
                            flags=A.QM_FLAG_WASM_SCAN_SEMANTICS)
        g, r = run_both(ctx, cols, q)
        assert_same(g, r, ctx_msg=str(flt))


def test_bigint_thresholds(ctx):
    cols = {"i": np.arange(-50, 50, dtype=np.int64), "f": np.linspace(-5.5, 5.5, 100),
            "k": np.zeros(100, np.int32)}
    for flt in ([FilterOp("i", "gt", BigInt(7))], [FilterOp("f", "lte", BigInt(2))], [FilterOp("f", "eq", BigInt(0))],
                [FilterOp("i", "between", [BigInt(-3), 4.5])], [FilterOp("i", "lt", -2.5)]):
        q = QueryDescriptor(filters=flt, group_by=["k"], aggregates=[AggregateOp("count", "*")])
        g, r = run_both(ctx, cols, q)
        assert_same(g, r, ctx_msg=str(flt))


def test_unordered_flag_same_groups(ctx):
    cols = datagen.events(1_000_000, seed=21)
    q = datagen.events_query()
    q.flags = A.QM_FLAG_UNORDERED
    g = ctx.table(cols).run(q)
    q2 = datagen.events_query()
    r = oracle.run(cols, q2)
    assert_same(g, r, ordered=False)


def test_qmcb_roundtrip(ctx):
    from querymode_b200 import qmcb
    rng = np.random.default_rng(6)
    n = 10_000
    cols = {"k": Column(rng.integers(0, 9, n).astype(np.int32), rng.random(n) < 0.1),
            "v": rng.normal(size=n), "w": rng.integers(0, 10, n).astype(np.int64)}
    buf = qmcb.encode(cols)
    t = ctx.table_from_qmcb(buf)
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("sum", "w"),
                                                    AggregateOp("count", "*")])
    g = t.run(q, with_qmcb=True)
    r = oracle.run(cols, q)
    assert_same(g, r)
    dec = qmcb.decode(g.qmcb)
    assert dec.names == g.names
    assert np.array_equal(dec.column("sum_v").values, g.column("sum_v").values)


def test_device_resident_columns(ctx):
    import torch
    cols = datagen.events(2_000_000, seed=31)
    dev = {k: torch.from_numpy(v).cuda() for k, v in cols.items()}
    q = datagen.events_query()
    g = ctx.table(dev).run(q)
    r = oracle.run(cols, q)
    assert_same(g, r)


def test_operator_pipeline_matches_reference(ctx):
    """FilterOperator -> AggregateOperator over 4096-row batches (the
    reference's conformance harness shape) against the oracle."""
    from querymode_b200.operators import AggregateOperator, ArrayScanOperator, FilterOperator, drain_pipeline
    from querymode_b200.rows import result_to_rows
    cols = datagen.orders(300_000, seed=5)
    q = datagen.orders_query()
    agg_q = QueryDescriptor(group_by=q.group_by, aggregates=q.aggregates)
    op = AggregateOperator(FilterOperator(ArrayScanOperator(cols, 4096), q.filters, ctx=ctx), agg_q, ctx=ctx)
    rows = drain_pipeline(op)
    ref = result_to_rows(oracle.run(cols, q, batch_rows=4096), True)
    assert [r["region"] for r in rows] == [r["region"] for r in ref]
    for a, b in zip(rows, ref):
        assert a["count_*"] == b["count_*"]
        assert abs(a["sum_amount"] - b["sum_amount"]) <= 1e-12 * abs(b["sum_amount"])
    # standalone FilterOperator narrows selections on the GPU
    f = FilterOperator(ArrayScanOperator(cols, 4096), q.filters, ctx=ctx)
    n = 0
    while (b := f.next_columnar()) is not None:
        n += b.selection.size
    assert n == int((cols["status"] == 1).sum())
    # an aggregation with no matching row: [{}] (reference finalize quirk)
    empty = AggregateOperator(FilterOperator(ArrayScanOperator(cols, 4096), [FilterOp("status", "eq", 9)], ctx=ctx),
                              agg_q, ctx=ctx)
    assert drain_pipeline(empty) == [{}]


@pytest.mark.parametrize("seed", range(8))
def test_filter_select_with_selection(ctx, seed):
    rng = np.random.default_rng(9000 + seed)
    n = int(rng.choice([1000, 70000]))
    cols = make_table(rng, n=n)
    q = rand_query(rng)
    sel = np.nonzero(rng.random(n) < 0.6)[0].astype(np.uint32)
    assert ctx.filter_select(cols, q, sel).tolist() == oracle.filter_select(cols, q, sel).tolist()


@pytest.mark.parametrize("depth", [2, 3])
def test_staged_filter_columns(ctx, depth):
    """The bulk-copy staged variant of the scan (opt-in) against the oracle."""
    cols = datagen.events(3_000_000, seed=17)
    q = datagen.events_query()
    ctx.set_tuning(local_slots=512, dedupe=0, stage_depth=depth)
    try:
        g = ctx.table(cols).run(q)
    finally:
        ctx.set_tuning()
    assert_same(g, oracle.run(cols, q))
    rng = np.random.default_rng(depth)
    n = 400_000
    c2 = {"k": Column(rng.integers(0, 300, n).astype(np.int64), rng.random(n) < 0.05),
          "x": Column(rng.normal(size=n), rng.random(n) < 0.1), "y": rng.integers(-5, 5, n).astype(np.int32)}
    q2 = QueryDescriptor(filters=[FilterOp("x", "gt", -0.5), FilterOp("y", "neq", 0)], group_by=["k"],
                         aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "*"), AggregateOp("max", "y")])
    ctx.set_tuning(stage_depth=depth)
    try:
        g2 = ctx.table(c2).run(q2)
    finally:
        ctx.set_tuning()
    assert_same(g2, oracle.run(c2, q2))


def test_per_warp_tables_large(ctx):
    # past the size where small direct tables (and the single no-GROUP-BY
    # slot) are copied per warp and updated without atomics
    rng = np.random.default_rng(21)
    n = 9_000_000
    x = rng.normal(size=n) * 100
    x[rng.random(n) < 0.001] = 0.0
    x[rng.random(n) < 0.001] = -0.0
    x[rng.random(n) < 1e-5] = math.nan
    cols = {"k": Column(rng.integers(0, 12, n).astype(np.int32), rng.random(n) < 0.02),
            "x": Column(x, rng.random(n) < 0.05),
            "i": rng.integers(-2**62, 2**62, n).astype(np.int64),
            "j": rng.integers(-2**31, 2**31 - 1, n).astype(np.int32),
            "f": rng.integers(0, 100, n).astype(np.int32)}
    aggs = [AggregateOp("sum", "x"), AggregateOp("min", "x"), AggregateOp("max", "x"), AggregateOp("avg", "x"),
            AggregateOp("count", "x"), AggregateOp("sum", "i"), AggregateOp("avg", "i"), AggregateOp("min", "i"),
            AggregateOp("sum", "j"), AggregateOp("max", "j"), AggregateOp("count", "*")]
    t = ctx.table(cols)
    try:
        for dedupe in (-1, 1):  # planner's choice; warp deduplication (per-warp copies) forced
            ctx.set_tuning(dedupe=dedupe)
            for q in (QueryDescriptor(filters=[FilterOp("f", "lt", 70)], group_by=["k"], aggregates=aggs),
                      QueryDescriptor(filters=[FilterOp("f", "gte", 10)], aggregates=aggs)):
                g = t.run(q)
                r = oracle.run(cols, q, threads=8)
                assert_same(g, r, ctx_msg=f"dedupe={dedupe}")
    finally:
        ctx.set_tuning()


def test_selective_filter_sampled_estimate(ctx):
    # a selective filter over a wide key range: the group table is sized from
    # a strided sample of the predicate (and a sparse dense range turns into
    # a hash table); sorted and clustered filter columns included
    rng = np.random.default_rng(33)
    n = 3_000_000
    cols = {"key": rng.integers(0, 1 << 22, n).astype(np.int64),
            "flag": (rng.random(n) < 0.01).astype(np.int32),
            "ts": np.sort(rng.integers(0, 1 << 40, n)).astype(np.int64),
            "v": rng.normal(size=n)}
    t = ctx.table(cols)
    qs = [QueryDescriptor(filters=[FilterOp("flag", "eq", 1)], group_by=["key"],
                          aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("ts", "lt", int(cols["ts"][n // 50]))], group_by=["key"],
                          aggregates=[AggregateOp("max", "v"), AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("ts", "gte", int(cols["ts"][n - n // 30]))], group_by=["key"],
                          aggregates=[AggregateOp("min", "v"), AggregateOp("avg", "v")])]
    for q in qs:
        g = t.run(q)
        assert_same(g, oracle.run(cols, q, threads=8))
        assert g.stats.retries == 0
        assert g.stats.table_capacity <= 18  # a hash table of at most 2^18 slots


@pytest.mark.parametrize("shards", [2, 3])
def test_sharded_partials_merge_to_whole_table(ctx, shards):
    # the multi-GPU exchange on one GPU: each shard through its own
    # aggregation, partial rows exported with global row offsets and merged
    # into the first shard's aggregation, against the whole table
    import torch
    from querymode_b200.distributed import shard_range
    rng = np.random.default_rng(50 + shards)
    n = 600_000
    cols = {"k": Column(rng.integers(-5000, 5000, n).astype(np.int64), rng.random(n) < 0.01),
            "x": Column(rng.normal(size=n) * 10, rng.random(n) < 0.05),
            "i": rng.integers(-2**62, 2**62, n).astype(np.int64),
            "j": rng.integers(-1000, 1000, n).astype(np.int32)}
    cols["x"].values[rng.random(n) < 0.001] = -0.0
    qs = [QueryDescriptor(filters=[FilterOp("j", "gt", -500)], group_by=["k"],
                          aggregates=[AggregateOp("sum", "x"), AggregateOp("min", "x"), AggregateOp("max", "x"),
                                      AggregateOp("avg", "i"), AggregateOp("sum", "i"), AggregateOp("count", "*"),
                                      AggregateOp("count", "x"), AggregateOp("max", "j")]),
          QueryDescriptor(filters=[FilterOp("j", "lt", 100)],
                          aggregates=[AggregateOp("sum", "i"), AggregateOp("min", "x"), AggregateOp("count", "*")])]
    for q in qs:
        streams = []
        parts = []
        for r in range(shards):
            a, b = shard_range(n, r, shards)
            shard = {k: (Column(v.values[a:b], v.nulls[a:b]) if isinstance(v, Column) else v[a:b])
                     for k, v in cols.items()}
            s = ctx.aggregate(q)
            s.push(shard)
            parts.append(s.export_partial(a))
            streams.append(s)
        for p in parts[1:]:
            streams[0].merge_partial(p, n)
        g = streams[0].finish()
        ref = oracle.run(cols, q)
        assert_same(g, ref)
        # the same through registered shard tables (push_table)
        tables = []
        for r in range(shards):
            a, b = shard_range(n, r, shards)
            tables.append(ctx.table({k: (Column(v.values[a:b], v.nulls[a:b]) if isinstance(v, Column) else v[a:b])
                                     for k, v in cols.items()}))
        aggs = [ctx.aggregate(q) for _ in range(shards)]
        for t, s in zip(tables, aggs):
            s.push_table(t)
        rows = [s.export_partial(shard_range(n, r, shards)[0]) for r, s in enumerate(aggs)]
        for p in rows[1:]:
            aggs[0].merge_partial(p, n)
        assert_same(aggs[0].finish(), ref)
        torch.cuda.synchronize()


def test_large_dense_table_key_range_passes(ctx):
    # a dense key range whose group table exceeds the L2 budget is updated in
    # key-range passes (each row once; NULL keys in the first pass only)
    rng = np.random.default_rng(61)
    n = 5_000_000
    cols = {"k": Column(rng.integers(0, 2_500_000, n).astype(np.int64), rng.random(n) < 0.001),
            "x": rng.normal(size=n), "f": rng.integers(0, 10, n).astype(np.int32)}
    t = ctx.table(cols)
    for q in (QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "*"),
                                                          AggregateOp("max", "x")]),
              QueryDescriptor(filters=[FilterOp("f", "lt", 9)], group_by=["k"],
                              aggregates=[AggregateOp("avg", "x"), AggregateOp("count", "*")])):
        g = t.run(q)
        assert g.stats.strategy in (0, 1, 2)
        assert_same(g, oracle.run(cols, q, threads=8))


def test_zone_maps_skip_zones_exactly(ctx):
    # sorted / clustered filter columns let whole 65,536-row zones be skipped;
    # the result must equal a scan of every row
    rng = np.random.default_rng(71)
    n = 3_000_000
    ts = np.sort(rng.integers(0, 10**12, n)).astype(np.int64)
    f = np.repeat(rng.normal(size=n // 1000), 1000)[:n] * 100
    f = np.concatenate([f, np.zeros(n - len(f))])
    cols = {"ts": Column(ts, rng.random(n) < 0.001), "f": f,
            "c": (np.arange(n) // 70_000).astype(np.int32),
            "k": rng.integers(0, 5000, n).astype(np.int64), "v": rng.normal(size=n)}
    t = ctx.table(cols)
    cut = int(ts[n // 3]), int(ts[n // 3 + 200_000])
    qs = [QueryDescriptor(filters=[FilterOp("ts", "gte", cut[0]), FilterOp("ts", "lt", cut[1])], group_by=["k"],
                          aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("c", "eq", 7)], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("c", "neq", 7)], group_by=["c"], aggregates=[AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("f", "gt", 250.0)], group_by=["k"], aggregates=[AggregateOp("max", "v")]),
          QueryDescriptor(filter_groups=[[FilterOp("c", "eq", 3)], [FilterOp("c", "between", [30, 31])]],
                          group_by=["c"], aggregates=[AggregateOp("count", "*"), AggregateOp("min", "ts")]),
          QueryDescriptor(filters=[FilterOp("ts", "is_null")], aggregates=[AggregateOp("count", "*")]),
          QueryDescriptor(filters=[FilterOp("ts", "gt", 10**13)], aggregates=[AggregateOp("count", "*")])]
    for q in qs:
        assert_same(t.run(q), oracle.run(cols, q, threads=8))


def test_large_hash_table_update_passes(ctx):
    # a hash table far beyond L2 (4M slots), with a NULL key and a key equal
    # to the empty-slot sentinel (both in reserved slots)
    rng = np.random.default_rng(81)
    n = 20_000_000
    universe = rng.integers(-2**62, 2**62, 1_000_000).astype(np.int64)
    universe[7] = np.iinfo(np.int64).min
    key = universe[rng.integers(0, len(universe), n)]
    cols = {"k": Column(key, rng.random(n) < 0.001), "x": rng.normal(size=n),
            "f": rng.integers(0, 10, n).astype(np.int32)}
    t = ctx.table(cols)
    for q in (QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "*")]),
              QueryDescriptor(filters=[FilterOp("f", "lt", 8)], group_by=["k"],
                              aggregates=[AggregateOp("max", "x"), AggregateOp("count", "*")])):
        g = t.run(q)
        assert g.stats.retries == 0
        assert_same(g, oracle.run(cols, q, threads=16))
        assert g.stats.rows_selected == (n if not q.filters else int((cols["f"] < 8).sum()))


def test_tables_recycle_device_blocks(ctx):
    # tables created and dropped in turn reuse each other's device blocks
    # (sizes within a quarter of each other); every table must see only its
    # own cells and NULLs
    rng = np.random.default_rng(91)
    q = QueryDescriptor(filters=[FilterOp("f", "gte", 0)], group_by=["k"],
                        aggregates=[AggregateOp("sum", "x"), AggregateOp("count", "x"), AggregateOp("min", "f")])
    for it in range(6):
        n = 1_000_000 + int(rng.integers(0, 200_000))
        cols = {"k": rng.integers(0, 50, n).astype(np.int32),
                "x": Column(rng.normal(size=n), rng.random(n) < (0.3 if it % 2 else 0.0) + 1e-9),
                "f": Column(rng.integers(-5, 100, n).astype(np.int64), rng.random(n) < 0.05 * (it % 3))}
        t = ctx.table(cols)
        assert_same(t.run(q), oracle.run(cols, q), ctx_msg=f"table {it}")
        t.close()
    assert ctx.trim() > 0  # the last table's blocks were kept
    assert ctx.trim() == 0


def test_statistics_at_upload_match_lazy_ones(ctx):
    # a host table of >= 4M rows gets its min / max, max |x| and zone maps
    # while it uploads; the same columns borrowed from device memory get them
    # on first use; both must plan to the oracle's results
    import torch
    rng = np.random.default_rng(101)
    n = 5_000_000
    ts = np.sort(rng.integers(0, 10**12, n)).astype(np.int64)
    plain = {"ts": ts, "k": rng.integers(-300, 4000, n).astype(np.int32), "v": rng.normal(size=n) * 1e6,
             "f": rng.random(n).astype(np.float32)}
    nullable = dict(plain, ts=Column(ts, rng.random(n) < 0.001), v=Column(plain["v"], rng.random(n) < 0.01))
    cut = int(ts[n // 4]), int(ts[n // 4 + 300_000])
    qs = [QueryDescriptor(filters=[FilterOp("ts", "gte", cut[0]), FilterOp("ts", "lt", cut[1])], group_by=["k"],
                          aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*"), AggregateOp("max", "f")]),
          QueryDescriptor(filters=[FilterOp("f", "lt", 0.5)], group_by=["k"],
                          aggregates=[AggregateOp("sum", "v"), AggregateOp("min", "ts"), AggregateOp("avg", "f")]),
          QueryDescriptor(filters=[FilterOp("v", "gt", 1e6)], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])]
    dev = {k: torch.from_numpy(v).cuda() for k, v in plain.items()}
    tables = [("host", ctx.table(plain), plain), ("borrowed", ctx.table(dev), plain),
              ("host with NULLs", ctx.table(nullable), nullable)]
    for name, t, cols in tables:
        for q in qs:
            assert_same(t.run(q), oracle.run(cols, q, threads=8), ctx_msg=name)
        t.close()


def test_large_pageable_columns_staged(ctx):
    # host columns of >= 64 MB in pageable memory go through pinned staging
    # buffers filled by host threads; the table must hold the same cells
    rng = np.random.default_rng(111)
    n = 9_000_000
    cols = {"k": rng.integers(0, 1000, n).astype(np.int64), "v": rng.normal(size=n),
            "f": Column(rng.integers(0, 100, n).astype(np.int64), rng.random(n) < 0.01)}
    t = ctx.table(cols)
    q = QueryDescriptor(filters=[FilterOp("f", "lt", 50)], group_by=["k"],
                        aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*"), AggregateOp("max", "f")])
    assert_same(t.run(q), oracle.run(cols, q, threads=8))
    t.close()


def test_corrupt_qmcb_refused_or_decoded(ctx):
    # byte flips and truncations of a QMCB buffer: each call builds a table or
    # returns QM_ERR_INVALID / UNSUPPORTED, never reads past the buffer; a table
    # it builds holds the cells the host decoder reads from the same bytes
    from querymode_b200 import _abi as A
    from querymode_b200 import qmcb
    rng = np.random.default_rng(41)
    n = 500
    cols = {"k": Column(rng.integers(0, 9, n).astype(np.int32), rng.random(n) < 0.1),
            "v": rng.normal(size=n), "w": rng.integers(0, 10, n).astype(np.int64)}
    buf = qmcb.encode(cols)
    built = compared = 0
    for trial in range(200):
        b = bytearray(buf)
        for _ in range(int(rng.integers(1, 4))):
            b[int(rng.integers(0, 40 if trial % 2 else len(b)))] = int(rng.integers(0, 256))
        if trial % 5 == 0:
            b = b[:int(rng.integers(1, len(b)))]
        try:
            t = ctx.table_from_qmcb(bytes(b))
        except A.QmError as e:
            assert e.status in (A.QM_ERR_INVALID, A.QM_ERR_UNSUPPORTED)
            continue
        except (ValueError, UnicodeDecodeError):
            continue
        built += 1
        try:
            dec = qmcb.decode(bytes(b))
        except Exception:
            t.close()
            continue
        for i, name in enumerate(t.names):
            if name in dec.names:
                vals, nulls = t.read_column(name)
                want = dec.column(name)
                assert np.array_equal(vals.view(np.uint8), np.asarray(want.values).view(np.uint8)), name
                compared += 1
        t.close()
    assert built > 0 and compared > 0


def test_retries_after_stale_statistics(ctx):
    # borrowed device columns rewritten in place after their statistics were
    # cached: the next query plans a direct range the keys leave (retry as a
    # hash table), then a hash table too small for them (retry larger); the
    # small result takes the one-synchronise path, whose failed attempts must
    # be discarded, and the answer must equal the oracle's on the new data
    import torch
    rng = np.random.default_rng(121)
    n = 400_000
    k0 = rng.integers(0, 100, n).astype(np.int64)
    v = rng.normal(size=n)
    dk = torch.from_numpy(k0).cuda()
    t = ctx.table({"k": dk, "v": torch.from_numpy(v).cuda()})
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    assert_same(t.run(q), oracle.run({"k": k0, "v": v}, q))
    k1 = rng.integers(-1000, 2000, n).astype(np.int64)
    dk.copy_(torch.from_numpy(k1))
    g = t.run(q)
    assert g.stats.retries >= 1, g.stats
    assert_same(g, oracle.run({"k": k1, "v": v}, q))
    t.close()
