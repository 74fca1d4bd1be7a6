"""qm_query_run_noalloc: the GROUP BY for callers that cannot allocate device
memory (code living inside another framework's memory arena, or where
cudaMalloc is not available to it).  It keeps every temporary in a fixed
static device array, so its results must equal qm_query_run's on the same
input — checked here on two calls in a row (the second call reuses the array
the first one left behind).  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import oracle
from querymode_b200 import _abi as A
from querymode_b200 import datagen
from querymode_b200.engine import Result, ResultColumn, _ColumnSet, unpack_nulls
from querymode_b200.query import AggregateOp, CQuery, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu

_NP = {A.QM_I32: np.int32, A.QM_I64: np.int64, A.QM_F64: np.float64}


def run_noalloc(ctx, dev_cols, q, max_groups, names_keys):
    import torch
    cs = _ColumnSet(dev_cols)
    cq = CQuery(q)
    n_out = len(names_keys)
    outs = [torch.full((max_groups * 16,), 0xAB, dtype=torch.uint8, device="cuda") for _ in range(n_out)]
    nulls = [torch.full(((max_groups + 31) // 32,), -1, dtype=torch.int32, device="cuda") for _ in range(n_out)]
    ptrs = (C.c_void_p * n_out)(*[o.data_ptr() for o in outs])
    nptrs = (C.c_void_p * n_out)(*[x.data_ptr() for x in nulls])
    dtypes = (C.c_int32 * n_out)()
    groups = C.c_int64()
    st = ctx.lib.qm_query_run_noalloc(ctx.h, cs.n_rows, cs.count, cs.array, cq.ref, max_groups, ptrs, nptrs,
                                      dtypes, C.byref(groups))
    ctx.check(st)
    G = groups.value
    cols = []
    for k, (name, is_key) in enumerate(names_keys):
        dt = dtypes[k]
        size = 16 if dt == A.QM_I128 else np.dtype(_NP[dt]).itemsize
        raw = outs[k][: G * size].cpu().numpy()
        vals = raw.view(np.int64).reshape(G, 2) if dt == A.QM_I128 else raw.view(_NP[dt])
        words = nulls[k][: (G + 31) // 32].cpu().numpy()
        mask = unpack_nulls(words.view(np.uint8), G) if G else np.zeros(0, bool)
        cols.append(ResultColumn(name, dt, is_key, vals.copy(), mask if mask.any() else None))
    return Result(cols, G)


def test_noalloc_matches_query_run_on_two_calls(ctx):
    import torch
    cols = datagen.events(2_000_000, seed=41)
    q = datagen.events_query()
    ref = ctx.table(cols).run(q)
    dev = {k: torch.from_numpy(v).cuda() for k, v in cols.items()}
    names = [(c.name, c.is_key) for c in ref.columns]
    want = oracle.run(cols, q)
    for _ in range(2):
        got = run_noalloc(ctx, dev, q, 70_000, names)
        assert_same(got, ref, ordered=False)
        assert_same(got, want, ordered=False)


def test_noalloc_ungrouped_and_capacity_error(ctx):
    import torch
    rng = np.random.default_rng(8)
    n = 300_000
    cols = {"k": rng.integers(0, 5000, n).astype(np.int64), "v": rng.normal(size=n), "w": rng.integers(-9, 9, n).astype(np.int32)}
    dev = {k: torch.from_numpy(v).cuda() for k, v in cols.items()}
    q = QueryDescriptor(filters=[FilterOp("w", "gt", 0)],
                        aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*"), AggregateOp("min", "w")])
    ref = ctx.table(cols).run(q)
    for _ in range(2):
        got = run_noalloc(ctx, dev, q, 1, [(c.name, c.is_key) for c in ref.columns])
        assert_same(got, ref)
    qg = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "v")])
    with pytest.raises(A.QmError) as ei:
        run_noalloc(ctx, dev, qg, 100, [("k", True), ("sum_v", False)])
    assert ei.value.status == A.QM_ERR_CAPACITY
    with pytest.raises(A.QmError) as ei:
        run_noalloc(ctx, dev, qg, 1 << 26, [("k", True), ("sum_v", False)])
    assert ei.value.status == A.QM_ERR_CAPACITY


def test_noalloc_key_packing_limit(ctx):
    """Without column statistics two int64 group columns cannot be packed
    into one key word: QM_ERR_UNSUPPORTED (qm_query_run packs them by their
    value ranges); two non-NULL int32 columns concatenate and match the
    oracle."""
    import torch
    rng = np.random.default_rng(9)
    n = 100_000
    cols = {"a": rng.integers(0, 40, n).astype(np.int64), "b": rng.integers(0, 30, n).astype(np.int64),
            "c": rng.integers(-5, 5, n).astype(np.int32), "d": rng.integers(0, 9, n).astype(np.int32),
            "v": rng.normal(size=n)}
    dev = {k: torch.from_numpy(v).cuda() for k, v in cols.items()}
    q64 = QueryDescriptor(group_by=["a", "b"], aggregates=[AggregateOp("sum", "v")])
    with pytest.raises(A.QmError) as ei:
        run_noalloc(ctx, dev, q64, 4096, [("a", True), ("b", True), ("sum_v", False)])
    assert ei.value.status == A.QM_ERR_UNSUPPORTED
    q32 = QueryDescriptor(group_by=["c", "d"], aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*")])
    for _ in range(2):
        got = run_noalloc(ctx, dev, q32, 4096, [("c", True), ("d", True), ("sum_v", False), ("count_*", False)])
        assert_same(got, oracle.run(cols, q32), ordered=False)
    assert_same(ctx.table(cols).run(q64), oracle.run(cols, q64))
