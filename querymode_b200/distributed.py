"""Multi-GPU filter -> GROUP BY: one process per GPU, rows sharded by
contiguous ranges, partial group states exchanged once.

The reference fans a query out to fragment DOs, each computing a partial
aggregate over its fragments, and reduces the partials
(src/query-do.ts:1747-1887 fan-out, src/merge.ts:156-172 and
mergePartialAggs src/partial-agg.ts:277-304).  Here every rank streams its
shard through its own aggregation (the fused scan on its GPU), exports the
occupied group slots as partial rows with FIRST moved to global rows,
all-gathers the rows (NCCL over NVLink on GPUs; any torch.distributed
backend works) and the root merges them into its aggregation before the
finalize, so the result equals a single-GPU run over the whole table:
same groups, same first-seen order, exact integer aggregates, compensated
float sums.

The exchange is written against a small protocol (push / export_partial /
merge_partial / finish) that engine.AggStream implements, so its host logic
runs under gloo on CPU too.
"""
from __future__ import annotations

from typing import Protocol

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


def allgather_rows(rows: torch.Tensor, group=None) -> list[torch.Tensor]:
    """All-gather a [n_r, w] tensor whose row count differs per rank: the
    counts first, then every rank's rows padded to the largest count."""
    world = dist.get_world_size(group)
    n = torch.tensor([rows.shape[0]], dtype=torch.int64, device=rows.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    counts = [int(s.item()) for s in sizes]
    m = max(counts)
    pad = torch.zeros((m, rows.shape[1]), dtype=rows.dtype, device=rows.device)
    pad[: rows.shape[0]] = rows
    out = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return [o[:c] for o, c in zip(out, counts)]


def aggregate_sharded(agg: PartialAggregator, shard, row_offset: int, rows_total: int, group=None, root: int = 0):
    """Aggregate this rank's shard (its first global row is row_offset),
    exchange the partials and return the merged result on `root` (None on
    the other ranks).  Every rank takes the same collective steps.  The
    root's own shard must start at global row 0 (rank 0 of shard_range),
    since its own slots are not moved."""
    rank = dist.get_rank(group)
    if rank == root and row_offset != 0:
        raise ValueError("the root's shard must start at global row 0")
    if hasattr(shard, "h") and hasattr(agg, "push_table"):  # a registered, device-resident table
        agg.push_table(shard)
    else:
        agg.push(shard)
    parts = allgather_rows(agg.export_partial(row_offset), group)
    if rank != root:
        return None
    for r, p in enumerate(parts):
        if r != root:
            agg.merge_partial(p, rows_total)
    return agg.finish()
