"""QM_FLAG_DETERMINISTIC: float SUM / AVG as exact fixed-point integer sums.

Under the flag, the same query returns bit-identical float sums on every run:
alone, replayed, in batches of any wave split and launch mode, and in a
serving mix beside other requests.  The sums stay within the path's 1e-12
tolerance of the reference's sequential sum (tests/helpers.py), NaN and
Infinity cells included (src/partial-agg.ts:77: the reference's
`sum += v`).
"""
import numpy as np
import pytest

import oracle
from querymode_b200 import _abi as A
from querymode_b200 import datagen
from querymode_b200.engine import Column, Context
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu

DET = A.QM_FLAG_DETERMINISTIC


def det(q: QueryDescriptor) -> QueryDescriptor:
    q.flags |= DET
    return q


def float_cols(res):
    return {c.name: c.values.copy() for c in res.columns if c.dtype == A.QM_F64 and not c.is_key}


def assert_bits_equal(a, b, msg=""):
    fa, fb = float_cols(a), float_cols(b)
    assert fa.keys() == fb.keys()
    for k in fa:
        assert np.array_equal(fa[k].view(np.int64), fb[k].view(np.int64)), f"{msg} {k} differs bit-wise"


def cancelling_table(n=3_000_000, seed=5):
    """Mixed-sign values over 12 orders of magnitude under a hot key (Zipf):
    a float sum whose last bits depend on the order of the adds."""
    rng = np.random.default_rng(seed)
    mag = 10.0 ** rng.uniform(-6, 6, n)
    return {"k": (rng.zipf(1.3, n) % 3000).astype(np.int64), "v": mag * rng.choice([-1.0, 1.0], n),
            "f": rng.integers(0, 100, n).astype(np.int32)}


def query():
    return QueryDescriptor(filters=[FilterOp("f", "lt", 80)], group_by=["k"],
                           aggregates=[AggregateOp("sum", "v"), AggregateOp("avg", "v"), AggregateOp("count", "*"),
                                       AggregateOp("min", "v")])


def test_same_bits_every_run_and_within_tolerance(ctx):
    cols = cancelling_table()
    t = ctx.table(cols)
    q = det(query())
    first = t.run(q)
    assert_same(first, oracle.run(cols, q))
    for _ in range(4):
        assert_bits_equal(t.run(q), first, "rerun")
    # the launch shape does not change the bits either
    for tuning in ({"local_slots": -1}, {"dedupe": 1}, {"blocks_per_sm": 1}):
        ctx.set_tuning(**tuning)
        try:
            assert_bits_equal(t.run(q), first, f"tuning {tuning}")
        finally:
            ctx.set_tuning()


def test_batches_and_waves_keep_the_bits(ctx):
    cols = cancelling_table(1_500_000, seed=9)
    others = [datagen.batch_table(s) for s in datagen.batch_specs(12, seed=4, rows_lo=1e4, rows_hi=3e5)]
    t = ctx.table(cols)
    q = det(query())
    alone = t.run(q)
    handles = [t] + [ctx.table(o) for o in others]
    qs = [q] + [det(datagen.batch_query(s)) for s in datagen.batch_specs(12, seed=4, rows_lo=1e4, rows_hi=3e5)]
    alone_others = [h.run(x) for h, x in zip(handles[1:], qs[1:])]
    b = ctx.batch(handles, qs)
    try:
        for mode in (1, 0):
            b.set_mode(mode)
            for waves in (1, 3, 0):
                b.set_waves(waves)
                res = b.run()
                assert_bits_equal(res[0], alone, f"mode {mode} waves {waves}")
                for i, r in enumerate(alone_others):
                    assert_bits_equal(res[i + 1], r, f"mode {mode} waves {waves} query {i + 1}")
    finally:
        b.close()


def test_serving_mix_keeps_the_bits():
    ctx = Context(0)
    cols = cancelling_table(1_000_000, seed=13)
    t = ctx.table(cols)
    q = det(query())
    alone = t.run(q)
    small = ctx.table(datagen.orders(300_000, seed=2))
    sq = det(datagen.orders_query())
    small_alone = small.run(sq)
    srv = ctx.server(hbm_budget_bytes=8 << 30, max_batch=8, lanes=3)
    try:
        tickets = [(srv.submit(t, q), alone) if i % 3 == 0 else (srv.submit(small, sq), small_alone) for i in range(30)]
        for tk, want in tickets:
            res, _ = srv.wait(tk)
            assert_bits_equal(res, want, "in the serving mix")
    finally:
        srv.close()


def test_non_finite_cells_follow_the_reference(ctx):
    rng = np.random.default_rng(3)
    n = 200_000
    v = rng.normal(size=n) * 1e3
    k = rng.integers(0, 8, n).astype(np.int32)
    v[k == 1] = np.where(rng.random(int((k == 1).sum())) < 0.01, np.nan, v[k == 1])
    idx2 = np.flatnonzero(k == 2)
    v[idx2[:3]] = np.inf
    idx3 = np.flatnonzero(k == 3)
    v[idx3[:2]] = np.inf
    v[idx3[2:4]] = -np.inf
    idx4 = np.flatnonzero(k == 4)
    v[idx4[:5]] = -np.inf
    cols = {"k": k, "v": Column(v, rng.random(n) < 0.05)}
    q = det(QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("avg", "v"),
                                                        AggregateOp("count", "v")]))
    g = ctx.table(cols).run(q)
    assert_same(g, oracle.run(cols, q))
    s = dict(zip(g.column("k").values.tolist(), g.column("sum_v").values.tolist()))
    assert np.isnan(s[1]) and s[2] == np.inf and np.isnan(s[3]) and s[4] == -np.inf and np.isfinite(s[0])


def test_stale_statistics_rerun(ctx):
    """Borrowed device columns rewritten with larger values after their
    statistics were cached: the fixed-point range no longer holds, the kernel
    says so, and the query re-plans and re-runs to the oracle's answer."""
    import torch
    rng = np.random.default_rng(21)
    n = 400_000
    k = rng.integers(0, 50, n).astype(np.int64)
    v = rng.normal(size=n)
    dv = torch.from_numpy(v.copy()).cuda()
    t = ctx.table({"k": torch.from_numpy(k).cuda(), "v": dv})
    q = det(QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")]))
    assert_same(t.run(q), oracle.run({"k": k, "v": v}, q))
    v2 = v * 1e9
    dv.copy_(torch.from_numpy(v2))
    g = t.run(q)
    assert g.stats.retries >= 1
    assert_same(g, oracle.run({"k": k, "v": v2}, q))


def test_streams_refuse_the_flag(ctx):
    with pytest.raises(A.QmError) as e:
        ctx.aggregate(det(query()))
    assert e.value.status == A.QM_ERR_UNSUPPORTED
