"""Serving loop (qm_server_*): requests batched together return exactly
what each returns alone; HBM budget admission defers or refuses;
cancellation, bad descriptors and waits that time out fail only their own
request."""
import numpy as np
import pytest

import oracle
from querymode_b200 import _abi as A
from querymode_b200 import datagen
from querymode_b200.engine import Column, Context
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def workload(seed=3):
    rng = np.random.default_rng(seed)
    n = 120_000
    tables = {
        "orders": datagen.orders(400_000, seed=seed),
        "events": datagen.events(600_000, seed=seed, n_keys=5000),
        "wide": datagen.wide_keys(500_000, seed=seed, n_keys=1 << 16),
        "gen": datagen.generate_rows(300_000),
        "nulls": {"k": Column(rng.integers(0, 40, n).astype(np.int64), rng.random(n) < 0.05),
                  "x": Column(rng.normal(size=n), rng.random(n) < 0.2),
                  "y": rng.integers(-9, 9, n).astype(np.int32)},
    }
    queries = [
        ("orders", datagen.orders_query()),
        ("events", datagen.events_query(window_start_day=int(rng.integers(0, 300)))),
        ("events", datagen.events_query(window_start_day=int(rng.integers(0, 300)))),
        ("wide", datagen.wide_keys_query(True)),
        ("wide", datagen.wide_keys_query(False)),
        ("gen", QueryDescriptor(filters=[FilterOp("amount", "gt", 500)], group_by=["region", "category"],
                                aggregates=[AggregateOp("sum", "score"), AggregateOp("count", "*"),
                                            AggregateOp("max", "amount")])),
        ("nulls", QueryDescriptor(filters=[FilterOp("y", "gte", 0)], group_by=["k"],
                                  aggregates=[AggregateOp("avg", "x"), AggregateOp("count", "x"),
                                              AggregateOp("sum", "y")])),
        ("nulls", QueryDescriptor(aggregates=[AggregateOp("sum", "x"), AggregateOp("min", "y")])),
    ]
    return tables, queries


def test_alone_equals_in_mix():
    ctx = Context(0)
    tables, queries = workload()
    handles = {k: ctx.table(v) for k, v in tables.items()}
    order = [i % len(queries) for i in range(40)]
    alone = [handles[queries[i][0]].run(queries[i][1]) for i in range(len(queries))]
    srv = ctx.server(hbm_budget_bytes=8 << 30, max_batch=16, max_wait_us=2000)
    try:
        tickets = [srv.submit(handles[queries[i][0]], queries[i][1]) for i in order]
        sizes = []
        for i, t in zip(order, tickets):
            res, timing = srv.wait(t)
            assert_same(res, alone[i], ctx_msg=f"query {i} in the mix")
            sizes.append(timing["batch_size"])
            assert timing["total_us"] >= timing["run_us"] >= 0
        st = srv.stats()
        assert st["completed"] == len(order) and st["failed"] == 0
        assert max(sizes) > 1  # requests were batched together
        assert st["batches"] < len(order)
    finally:
        srv.close()
    # and alone equals the oracle
    for i in (0, 1, 5, 6):
        name, q = queries[i]
        assert_same(alone[i], oracle.run(tables[name], q))


def test_budget_defers_and_refuses():
    ctx = Context(0)
    tables, queries = workload(5)
    handles = {k: ctx.table(v) for k, v in tables.items()}
    resident = sum(c.nbytes for name in ("orders", "wide") for c in tables[name].values())
    # beside the two resident tables, room for two small requests per batch
    # and never for the high-cardinality one
    srv = ctx.server(hbm_budget_bytes=resident + (400 << 10), max_batch=8)
    try:
        small = [srv.submit(handles["orders"], queries[0][1]) for _ in range(6)]
        big = srv.submit(handles["wide"], datagen.wide_keys_query(False))
        for t in small:
            res, timing = srv.wait(t)
            assert res.n_rows == 16
        with pytest.raises(A.QmError) as e:
            srv.wait(big)
        assert e.value.status == A.QM_ERR_OOM
        st = srv.stats()
        assert st["refused"] == 1 and st["completed"] == 6
        assert st["resident_bytes"] == resident
        assert st["batches"] >= 3  # deferred into later batches by the budget
    finally:
        srv.close()


def test_cancel_bad_descriptor_and_timeout():
    ctx = Context(0)
    tables, queries = workload(7)
    handles = {k: ctx.table(v) for k, v in tables.items()}
    alone = handles["orders"].run(queries[0][1])
    # a long batching window keeps requests queued long enough to cancel
    srv = ctx.server(hbm_budget_bytes=8 << 30, max_batch=64, max_wait_us=300_000)
    try:
        ts = [srv.submit(handles["orders"], queries[0][1]) for _ in range(6)]
        bad = srv.submit(handles["orders"], QueryDescriptor(group_by=["no_such_column"],
                                                             aggregates=[AggregateOp("count", "*")]))
        assert srv.cancel(ts[1]) and srv.cancel(ts[4])
        assert not srv.cancel(12345678)
        for i, t in enumerate(ts):
            if i in (1, 4):
                with pytest.raises(A.QmError) as e:
                    srv.wait(t)
                assert e.value.status == A.QM_ERR_CANCELLED
            else:
                res, _ = srv.wait(t)
                assert_same(res, alone)
        with pytest.raises(A.QmError) as e:
            srv.wait(bad)
        assert e.value.status != A.QM_OK and "no_such_column" in str(e.value)
        # a wait that runs out leaves the request pending
        t = srv.submit(handles["orders"], queries[0][1])
        with pytest.raises(A.QmError) as e:
            srv.wait(t, timeout_s=1e-6)
        assert e.value.status == A.QM_ERR_TIMEOUT
        res, _ = srv.wait(t)
        assert_same(res, alone)
        st = srv.stats()
        assert st["cancelled"] == 2 and st["failed"] == 1
    finally:
        srv.close()


def test_batch_row_cap_keeps_results():
    # a batch stops taking requests once their rows would pass max_batch_rows
    # (a request larger than the cap runs alone); results are unchanged
    ctx = Context(0)
    tables, queries = workload(11)
    handles = {k: ctx.table(v) for k, v in tables.items()}
    alone = [handles[name].run(q) for name, q in queries]
    cap = 700_000
    srv = ctx.server(hbm_budget_bytes=8 << 30, max_batch=64, max_wait_us=50_000, max_batch_rows=cap)
    try:
        order = [i % len(queries) for i in range(24)]
        tickets = [srv.submit(handles[queries[i][0]], queries[i][1]) for i in order]
        for i, t in zip(order, tickets):
            res, timing = srv.wait(t)
            assert_same(res, alone[i])
            rows = handles[queries[i][0]].n_rows
            assert timing["batch_size"] == 1 or rows <= cap
        assert srv.stats()["batches"] > 24 * 400_000 // cap // 4
    finally:
        srv.close()


def test_request_overlaps_heavy_batch():
    """A light request submitted while a heavy request (a 16.7M-group
    aggregate over 40M rows, run alone) is on the GPU starts on another lane
    at once and completes first; both equal their results alone."""
    import time
    ctx = Context(0)
    heavy_t = ctx.table(datagen.wide_keys(40_000_000, seed=31, n_keys=1 << 24))
    light_t = ctx.table(datagen.orders(400_000, seed=31))
    hq, lq = datagen.wide_keys_query(False), datagen.orders_query()
    heavy_alone, light_alone = heavy_t.run(hq), light_t.run(lq)
    srv = ctx.server(hbm_budget_bytes=40 << 30, max_batch=16, max_batch_rows=10_000_000, lanes=3)
    try:
        for _ in range(2):  # warm: buffers of both shapes on every lane
            for t in [srv.submit(heavy_t, hq), srv.submit(light_t, lq)]:
                srv.wait(t)
        h = srv.submit(heavy_t, hq)
        time.sleep(0.002)  # the heavy request is on the GPU
        t0 = time.perf_counter()
        lt = srv.submit(light_t, lq)
        lres, ltm = srv.wait(lt)
        light_s = time.perf_counter() - t0
        with pytest.raises(A.QmError) as e:  # the heavy request is still running
            srv.wait(h, timeout_s=1e-6)
        assert e.value.status == A.QM_ERR_TIMEOUT
        hres, htm = srv.wait(h)
        assert_same(lres, light_alone)
        assert_same(hres, heavy_alone)
        assert ltm["batch_size"] == 1 and htm["batch_size"] == 1
        assert light_s * 1e6 < htm["total_us"]
        st = srv.stats()
        assert st["heavy"] >= 3 and st["lanes"] == 3 and st["peak_in_flight"] >= 2
    finally:
        srv.close()


def test_planned_groups_make_a_request_heavy():
    """With max_batch_groups, a request the planner sizes at more groups (a
    16M-key aggregate over a table small enough to batch by rows) is sent
    back and runs alone on a lane that takes heavy requests; the light
    requests submitted with it still batch together; all equal their
    results alone."""
    ctx = Context(0)
    heavy_t = ctx.table(datagen.wide_keys(8_000_000, seed=32, n_keys=1 << 24))
    light_t = ctx.table(datagen.orders(300_000, seed=32))
    hq, lq = datagen.wide_keys_query(False), datagen.orders_query()
    heavy_alone, light_alone = heavy_t.run(hq), light_t.run(lq)
    srv = ctx.server(hbm_budget_bytes=40 << 30, max_batch=16, max_batch_rows=0, lanes=2, max_batch_groups=1 << 20)
    try:
        for _ in range(3):
            tickets = [srv.submit(light_t, lq) for _ in range(6)] + [srv.submit(heavy_t, hq)] + \
                      [srv.submit(light_t, lq) for _ in range(6)]
            timings = []
            for i, t in enumerate(tickets):
                res, tm = srv.wait(t)
                assert_same(res, heavy_alone if i == 6 else light_alone)
                timings.append(tm)
            assert timings[6]["batch_size"] == 1
        # (whether the request was sent back or a lane took it alone first
        # depends on timing; either way it ran alone)
        st = srv.stats()
        assert st["failed"] == 0
    finally:
        srv.close()
