"""Multi-GPU filter -> GROUP BY: one process per GPU, rows sharded by
contiguous ranges, partial group states exchanged once.

The reference fans a query out to fragment DOs, each computing a partial
aggregate over its fragments, and reduces the partials
(src/query-do.ts:1747-1887 fan-out, src/query-do.ts:1896-1960 and
src/merge.ts:156-172 reduce, mergePartialAggs src/partial-agg.ts:277-304).
Here every rank streams its shard through its own aggregation (the fused
scan on its GPU) and exports the occupied group slots as partial rows with
FIRST moved to global rows.  Then one of two exchanges:

* aggregate_sharded (few groups): the rows are gathered to the root, which
  merges them into its aggregation and finalizes;
* aggregate_partitioned (many groups): each rank splits its rows by the hash
  of the group key (qm_partial_partition), an all-to-all sends every part to
  its rank (grouped NCCL send / receive on GPUs), and each rank merges and
  finalizes the groups of its key range only.  Its result rows come in
  ascending order of their first global row; an ordered gather merges the
  ranks' results into the global first-seen order on the root.

Either way the result equals a single-GPU run over the whole table: same
groups, same first-seen order, exact integer aggregates, compensated float
sums.  The collectives work on any torch.distributed backend (gloo moves
host copies), so the host logic also runs on CPU; every rank takes the same
collective steps in the same order.
"""
from __future__ import annotations

from typing import Protocol

import numpy as np
import torch
import torch.distributed as dist


class PartialAggregator(Protocol):
    def push(self, columns) -> None: ...

    def export_partial(self, row_offset: int = 0) -> torch.Tensor: ...

    def merge_partial(self, rows: torch.Tensor, rows_end: int) -> None: ...

    def finish(self): ...


def shard_range(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [start, end) of `rank`: contiguous ranges, sizes differing by at
    most one, in rank order (rank r's rows precede rank r+1's)."""
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _wire(t: torch.Tensor, group) -> torch.Tensor:
    """The tensor on the device the group's backend moves (host for gloo)."""
    return t.cpu() if dist.get_backend(group) == "gloo" else t


def _counts_device(group) -> torch.device:
    if dist.get_backend(group) == "gloo":
        return torch.device("cpu")
    return torch.device("cuda", torch.cuda.current_device())


def allgather_rows(rows: torch.Tensor, group=None) -> list[torch.Tensor]:
    """All-gather a [n_r, w] tensor whose row count differs per rank: the
    counts first, then every rank's rows padded to the largest count."""
    world = dist.get_world_size(group)
    x = _wire(rows, group)
    n = torch.tensor([x.shape[0]], dtype=torch.int64, device=x.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    counts = [int(s.item()) for s in sizes]
    m = max(counts)
    pad = torch.zeros((m,) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
    pad[: x.shape[0]] = x
    out = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return [o[:c].to(rows.device) for o, c in zip(out, counts)]


def gather_rows(rows: torch.Tensor, root: int = 0, group=None) -> list[torch.Tensor] | None:
    """Gather a [n_r, ...] tensor whose row count differs per rank to
    `root` (its list, in rank order; None elsewhere): counts, then the rows
    padded to the largest count.  Only the root receives: (world - 1) x less
    traffic than an all-gather."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    x = _wire(rows, group)
    n = torch.tensor([x.shape[0]], dtype=torch.int64, device=x.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)  # every rank needs the pad size
    counts = [int(s.item()) for s in sizes]
    m = max(counts)
    pad = torch.zeros((m,) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
    pad[: x.shape[0]] = x
    out = [torch.empty_like(pad) for _ in range(world)] if rank == root else None
    dist.gather(pad, out, dst=root, group=group)
    if rank != root:
        return None
    return [o[:c].to(rows.device) for o, c in zip(out, counts)]


def alltoall_rows(rows: torch.Tensor, counts: list[int], group=None) -> torch.Tensor:
    """rows holds counts[r] rows for rank r, in rank order; returns the rows
    every rank sent to this one, in source-rank order (one all-to-all of the
    counts, one of the rows: grouped send / receive)."""
    x = _wire(rows, group)
    w = x.shape[1]
    send = torch.tensor(counts, dtype=torch.int64, device=_counts_device(group))
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    rcounts = [int(c) for c in recv.tolist()]
    out = torch.empty((sum(rcounts), w), dtype=x.dtype, device=x.device)
    dist.all_to_all_single(out, x.contiguous(), output_split_sizes=rcounts, input_split_sizes=list(counts),
                           group=group)
    return out.to(rows.device)


def _push(agg, shard) -> None:
    if hasattr(shard, "h") and hasattr(agg, "push_table"):  # a registered, device-resident table
        agg.push_table(shard)
    else:
        agg.push(shard)


def aggregate_sharded(agg: PartialAggregator, shard, row_offset: int, rows_total: int, group=None, root: int = 0):
    """Aggregate this rank's shard (its first global row is row_offset),
    gather the partials to `root` and return the merged result there (None
    on the other ranks).  The root's own shard must start at global row 0
    (rank 0 of shard_range), since its own slots are not moved."""
    rank = dist.get_rank(group)
    if rank == root and row_offset != 0:
        raise ValueError("the root's shard must start at global row 0")
    _push(agg, shard)
    parts = gather_rows(agg.export_partial(row_offset), root, group)
    if rank != root:
        return None
    for r, p in enumerate(parts):
        if r != root:
            agg.merge_partial(p, rows_total)
    return agg.finish()


class KeyRange:
    """One rank's share of a key-partitioned aggregate: the finished result
    of its key range (rows in ascending order of `first`, their groups'
    first global rows)."""

    def __init__(self, result, first: np.ndarray):
        self.result = result
        self.first = first


def aggregate_partitioned(agg, shard, row_offset: int, rows_total: int, partition, group=None,
                          root: int | None = 0):
    """Aggregate this rank's shard, exchange the partials by key (each rank
    receives every rank's rows of its key range), merge and finalize this
    rank's key range.  `partition(rows, parts)` splits partial rows into
    parts (Context.partition_partial on GPUs).  Returns this rank's KeyRange;
    with root set, the ranks' results are also gathered to the root in
    global first-seen order, which the root returns instead (other ranks:
    None)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    _push(agg, shard)
    rows = agg.export_partial(row_offset)
    sorted_rows, counts = partition(rows, world)
    mine = agg.partial_begin()
    try:
        recv = alltoall_rows(sorted_rows, counts, group)
        mine.merge_partial(recv, rows_total)
        _, first_word = mine.partial_layout()
        merged = mine.export_partial(0)
        first = np.sort(merged[:, first_word].cpu().numpy()) if first_word >= 0 else np.arange(merged.shape[0])
        local = KeyRange(mine.finish(), first)
    finally:
        mine.close()
    if root is None:
        return local
    union = ordered_gather(local, root, group)
    return union if rank == root else None


def merge_key_ranges(parts: list[tuple[np.ndarray, list]]):
    """The global first-seen order of key-range results: parts are (first
    global rows, columns) per rank, each rank's columns a list of
    (name, dtype, is_key, values, nulls); rows of all ranks ordered by their
    first global row (a group lives on one rank only, so nothing merges)."""
    from .engine import Result, ResultColumn
    order = np.argsort(np.concatenate([np.asarray(f, dtype=np.int64) for f, _ in parts]), kind="stable")
    out = []
    for k, (name, dtype, is_key, _, _) in enumerate(parts[0][1]):
        vals = np.concatenate([cols[k][3] for _, cols in parts])[order]
        nulls = np.concatenate([cols[k][4] if cols[k][4] is not None else np.zeros(len(cols[k][3]), bool)
                                for _, cols in parts])[order]
        out.append(ResultColumn(name, dtype, is_key, vals.copy(), nulls if nulls.any() else None))
    return Result(out, len(order))


def _columns(result) -> list:
    return [(c.name, c.dtype, c.is_key, np.ascontiguousarray(c.values), c.nulls) for c in result.columns]


def ordered_gather(local: KeyRange, root: int = 0, group=None):
    """The ranks' key-range results gathered to `root` and merged into the
    global first-seen order: every column is gathered as raw bytes with its
    NULL mask, then merge_key_ranges orders the rows by their first global
    rows.  Returns a Result on the root, None elsewhere."""
    rank = dist.get_rank(group)
    dev = _counts_device(group)
    firsts = gather_rows(torch.from_numpy(np.ascontiguousarray(local.first, dtype=np.int64)).to(dev), root, group)
    mine = _columns(local.result)
    gathered = []
    for name, dtype, is_key, v, nulls in mine:
        width = v.dtype.itemsize * int(np.prod(v.shape[1:], dtype=np.int64))
        raw = torch.from_numpy(v.view(np.uint8).reshape(len(v), width))
        nb = torch.from_numpy((nulls if nulls is not None else np.zeros(len(v), bool)).astype(np.uint8))
        gathered.append((gather_rows(raw.to(dev), root, group), gather_rows(nb.to(dev), root, group)))
    if rank != root:
        return None
    parts = []
    for r in range(len(firsts)):
        cols = []
        for (name, dtype, is_key, v, _), (raws, nbs) in zip(mine, gathered):
            vals = raws[r].cpu().numpy().reshape(-1).view(v.dtype).reshape((-1,) + v.shape[1:])
            cols.append((name, dtype, is_key, vals, nbs[r].cpu().numpy().astype(bool)))
        parts.append((firsts[r].cpu().numpy(), cols))
    return merge_key_ranges(parts)
