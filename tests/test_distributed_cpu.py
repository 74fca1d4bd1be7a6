"""The multi-GPU exchanges' host logic on CPU: world size 2 (and 3) over gloo
(127.0.0.1).  A numpy aggregator stands in for the GPU aggregation with the
same partial-row layout as AggStream.export_partial ([key word, special
flag, accumulator words], FIRST moved to global rows) and the same protocol
(push / export_partial / merge_partial / partial_begin / partial_layout /
finish); the sharding, the gather to the root, the key-partitioned
all-to-all and the ordered gather are the code the GPU path runs.  The GPU
versions of these tests (the library's own export, partition and merge)
are in tests/test_gpu_distributed.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from querymode_b200.distributed import (aggregate_partitioned, aggregate_sharded, allgather_rows, alltoall_rows,
                                        gather_rows, merge_key_ranges, shard_range)
from querymode_b200.engine import Result, ResultColumn

QM_I64 = 1


class DictAgg:
    """COUNT(*) and SUM(v) by k in first-seen order.  Partial rows are
    [key, special, count, first global row, sum] (FIRST is word 3)."""

    def __init__(self):
        self.state = {}
        self.offset = 0

    def push(self, shard):
        for i, (k, v) in enumerate(zip(shard["k"].tolist(), shard["v"].tolist())):
            c, f, s = self.state.get(k, (0, i, 0))
            self.state[k] = (c + 1, min(f, i), s + v)

    def export_partial(self, row_offset=0):
        rows = [[k, 0, c, f + row_offset, s] for k, (c, f, s) in self.state.items()]
        return torch.tensor(rows, dtype=torch.int64).reshape(-1, 5)

    def merge_partial(self, rows, rows_end):
        for k, _, c, f, s in rows.tolist():
            c0, f0, s0 = self.state.get(k, (0, f, 0))
            self.state[k] = (c0 + c, min(f0, f), s0 + s)

    def partial_begin(self):
        return DictAgg()

    def partial_layout(self):
        return 5, 3

    def close(self):
        pass

    def finish(self):
        rows = sorted(((f, k, c, s) for k, (c, f, s) in self.state.items()))
        col = lambda i: np.array([r[i] for r in rows], dtype=np.int64)
        return Result([ResultColumn("k", QM_I64, 1, col(1), None), ResultColumn("count", QM_I64, 0, col(2), None),
                       ResultColumn("sum", QM_I64, 0, col(3), None)], len(rows))


def partition(rows, parts):
    """Rows split by key into `parts` parts (part 0 first), with counts."""
    p = (rows[:, 0] % parts).numpy() if rows.shape[0] else np.zeros(0, np.int64)
    order = np.argsort(p, kind="stable")
    return rows[torch.from_numpy(order)], [int((p == i).sum()) for i in range(parts)]


def table(n, seed=3):
    rng = np.random.default_rng(seed)
    return {"k": rng.integers(-500, 500, n), "v": rng.integers(-10**9, 10**9, n)}


def expected(cols):
    agg = DictAgg()
    agg.push(cols)
    return agg.finish()


def same(a, b):
    assert a.n_rows == b.n_rows
    for x, y in zip(a.columns, b.columns):
        assert x.name == y.name and np.array_equal(x.values, y.values)


def _worker(rank, world, port, n, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # variable-size all-gather and gather
        mine = torch.arange(rank * 10, rank * 10 + 3 + 4 * rank, dtype=torch.int64).reshape(-1, 1)
        got = allgather_rows(mine)
        assert [g.shape[0] for g in got] == [3 + 4 * r for r in range(world)]
        assert torch.equal(got[rank], mine)
        g0 = gather_rows(mine, root=0)
        assert (g0 is None) == (rank != 0)
        if rank == 0:
            assert [g.shape[0] for g in g0] == [3 + 4 * r for r in range(world)]
        # all-to-all: rank r sends (r + 1) * (d + 1) rows tagged (r, d) to rank d
        counts = [(rank + 1) * (d + 1) for d in range(world)]
        rows = torch.tensor([[rank, d] for d in range(world) for _ in range(counts[d])], dtype=torch.int64)
        recv = alltoall_rows(rows, counts)
        want = [[r, rank] for r in range(world) for _ in range((r + 1) * (rank + 1))]
        assert recv.tolist() == want
        cols = table(n)
        a, b = shard_range(n, rank, world)
        shard = {k: v[a:b] for k, v in cols.items()}
        # few groups: gather to the root, merged there
        res = aggregate_sharded(DictAgg(), shard, a, n)
        if rank == 0:
            same(res, expected(cols))
        else:
            assert res is None
        # many groups: key-partitioned all-to-all, each rank its key range,
        # then the ordered gather
        kr = aggregate_partitioned(DictAgg(), shard, a, n, partition, root=None)
        assert np.all(np.diff(kr.first) > 0)
        assert all(k % world == rank for k in kr.result.column("k").values.tolist())
        res = aggregate_partitioned(DictAgg(), shard, a, n, partition, root=0)
        if rank == 0:
            same(res, expected(cols))
            open(os.path.join(out_dir, "ok"), "w").write("ok")
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,n", [(2, 10_001), (2, 7), (3, 5_000)])
def test_exchanges_gloo(tmp_path, world, n):
    mp.spawn(_worker, args=(world, _free_port(), n, str(tmp_path)), nprocs=world, join=True)
    assert (tmp_path / "ok").exists()


def test_merge_key_ranges_orders_by_first_row():
    cols = lambda k, c: [("k", QM_I64, 1, np.array(k), None), ("c", QM_I64, 0, np.array(c), np.array(c) < 0)]
    res = merge_key_ranges([(np.array([0, 7, 9]), cols([5, 1, 3], [1, -1, 2])),
                            (np.array([2, 3]), cols([8, 6], [4, 5])), (np.array([], np.int64), cols([], []))])
    assert res.column("k").values.tolist() == [5, 8, 6, 1, 3]
    assert res.column("c").nulls.tolist() == [False, False, False, True, False]


def test_shard_range_covers_rows_in_order():
    for n in (0, 1, 7, 100, 10_001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
