"""The multi-GPU exchange's host logic on CPU: world_size 2 over gloo
(127.0.0.1).  A numpy stand-in aggregator (COUNT, integer SUM, first-seen
order) replaces the GPU aggregation; the sharding, the variable-size
all-gather and the root merge are the code the GPU path runs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from querymode_b200.distributed import aggregate_sharded, allgather_rows, shard_range


class DictAgg:
    """COUNT(*) and SUM(v) by k in first-seen order; partial rows are
    [key, special, count, sum, first global row]."""

    def __init__(self):
        self.state = {}

    def push(self, shard):
        self.k, self.v = shard["k"], shard["v"]
        for i, (k, v) in enumerate(zip(self.k.tolist(), self.v.tolist())):
            c, s, f = self.state.get(k, (0, 0, i))
            self.state[k] = (c + 1, s + v, min(f, i))

    def export_partial(self, row_offset=0):
        rows = [[k, 0, c, s, f + row_offset] for k, (c, s, f) in self.state.items()]
        return torch.tensor(rows, dtype=torch.int64).reshape(-1, 5)

    def merge_partial(self, rows, rows_end):
        for k, _, c, s, f in rows.tolist():
            c0, s0, f0 = self.state.get(k, (0, 0, f))
            self.state[k] = (c0 + c, s0 + s, min(f0, f))

    def finish(self):
        return sorted(((f, k, c, s) for k, (c, s, f) in self.state.items()))


def table(n, seed=3):
    rng = np.random.default_rng(seed)
    return {"k": rng.integers(-50, 50, n), "v": rng.integers(-10**9, 10**9, n)}


def expected(cols):
    agg = DictAgg()
    agg.push(cols)
    return agg.finish()


def _worker(rank, world, port, n, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # variable-size all-gather
        mine = torch.arange(rank * 10, rank * 10 + 3 + 4 * rank, dtype=torch.int64).reshape(-1, 1)
        got = allgather_rows(mine)
        assert [g.shape[0] for g in got] == [3 + 4 * r for r in range(world)]
        assert torch.equal(got[rank], mine)
        # sharded aggregation, merged on rank 0
        cols = table(n)
        a, b = shard_range(n, rank, world)
        res = aggregate_sharded(DictAgg(), {k: v[a:b] for k, v in cols.items()}, a, n)
        if rank == 0:
            assert res == expected(cols)
            open(os.path.join(out_dir, "ok"), "w").write("ok")
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n", [10_001, 7])
def test_sharded_aggregate_gloo_world2(tmp_path, n):
    mp.spawn(_worker, args=(2, _free_port(), n, str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "ok").exists()


def test_shard_range_covers_rows_in_order():
    for n in (0, 1, 7, 100, 10_001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
