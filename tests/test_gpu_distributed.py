"""The multi-GPU exchanges with the library's own export, partition and merge
kernels, against the oracle over the whole table.

Every call here has one GPU, so the ranks are emulated: shards aggregate
independently (no kernel waits on another), their partial rows are split by
qm_partial_partition and exchanged, each key range is merged into its own
aggregation (qm_agg_partial_begin) and finalized, and the key ranges are
put back in global first-seen order.  Once in-process (the all-to-all as
list slicing), once as two processes on the GPU exchanging over gloo
through host memory (the code path of NCCL ranks, with host copies)."""
import os
import socket

import numpy as np
import pytest

import oracle
from querymode_b200.distributed import (KeyRange, aggregate_partitioned, aggregate_sharded, merge_key_ranges,
                                        shard_range)
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def table(n, seed):
    rng = np.random.default_rng(seed)
    cols = {"k": Column(rng.integers(-(1 << 40), 1 << 40, 1 << 17)[rng.integers(0, 1 << 17, n)].astype(np.int64),
                        rng.random(n) < 0.002),
            "x": Column(rng.normal(size=n) * 10, rng.random(n) < 0.05),
            "i": rng.integers(-2**62, 2**62, n).astype(np.int64),
            "j": rng.integers(-1000, 1000, n).astype(np.int32)}
    cols["x"].values[rng.random(n) < 0.001] = -0.0
    return cols


QUERY = QueryDescriptor(filters=[FilterOp("j", "gt", -700)], group_by=["k"],
                        aggregates=[AggregateOp("sum", "x"), AggregateOp("min", "x"), AggregateOp("max", "x"),
                                    AggregateOp("avg", "i"), AggregateOp("sum", "i"), AggregateOp("count", "*"),
                                    AggregateOp("count", "x"), AggregateOp("max", "j")])


def shard_of(cols, a, b):
    return {k: (Column(v.values[a:b], v.nulls[a:b]) if isinstance(v, Column) else v[a:b]) for k, v in cols.items()}


@pytest.mark.parametrize("world", [2, 3, 5])
def test_partitioned_exchange_in_process(ctx, world):
    n = 1_200_000
    cols = table(n, seed=60 + world)
    aggs, parts = [], []
    for r in range(world):
        a, b = shard_range(n, r, world)
        s = ctx.aggregate(QUERY)
        s.push(shard_of(cols, a, b))
        rows = s.export_partial(a)
        sorted_rows, counts = ctx.partition_partial(rows, world)
        assert sum(counts) == rows.shape[0]
        starts = np.concatenate([[0], np.cumsum(counts)])
        parts.append([sorted_rows[starts[d]:starts[d + 1]] for d in range(world)])
        aggs.append(s)
    import torch
    ranges, keys_seen = [], set()
    for d in range(world):
        mine = aggs[d].partial_begin()
        mine.merge_partial(torch.cat([parts[r][d] for r in range(world)]), n)
        _, fw = mine.partial_layout()
        first = np.sort(mine.export_partial(0)[:, fw].cpu().numpy())
        res = mine.finish()
        keys = set(res.column("k").values[~(res.column("k").nulls if res.column("k").nulls is not None
                                            else np.zeros(res.n_rows, bool))].tolist())
        assert not (keys & keys_seen)  # a group lives on one rank only
        keys_seen |= keys
        ranges.append(KeyRange(res, first))
        mine.close()
    got = merge_key_ranges([(kr.first, [(c.name, c.dtype, c.is_key, c.values, c.nulls) for c in kr.result.columns])
                            for kr in ranges])
    assert_same(got, oracle.run(cols, QUERY))
    for s in aggs:
        s.close()


def _worker(rank, world, port, n, out_dir):
    import torch
    import torch.distributed as dist

    from querymode_b200.engine import Context
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = Context(0)
    try:
        cols = table(n, seed=77)
        a, b = shard_range(n, rank, world)
        t = ctx.table(shard_of(cols, a, b))
        ref = oracle.run(cols, QUERY) if rank == 0 else None
        agg = ctx.aggregate(QUERY)
        res = aggregate_sharded(agg, t, a, n)
        agg.close()
        if rank == 0:
            assert_same(res, ref)
        agg = ctx.aggregate(QUERY)
        res = aggregate_partitioned(agg, t, a, n, ctx.partition_partial, root=0)
        agg.close()
        if rank == 0:
            assert_same(res, ref)
            open(os.path.join(out_dir, "ok"), "w").write("ok")
        t.close()
        torch.cuda.synchronize()
    finally:
        ctx.close()
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_exchanges_two_processes_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), 400_000, str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "ok").exists()
