"""The reference's pull-based operator API over the B200 path.

Mirrors ``Operator { next(): RowBatch | null; nextColumnar?(): ColumnarBatch |
null; close() }`` (src/operators.ts:67-75) with the two operators of the path:

* FilterOperator (src/operators.ts:1406-1496): narrows each batch's selection
  vector on the GPU (qm_filter_select);
* AggregateOperator (src/operators.ts:1646-1710): drains its upstream batch by
  batch into one streaming GPU aggregation (qm_agg_*), then yields all result
  rows once and None afterwards.  When its upstream is a FilterOperator the
  filter is fused into the aggregation kernel, as the reference's scan fuses
  its WASM filter ahead of the aggregate (src/operators.ts:3084).

A ColumnarBatch carries numpy arrays (or engine.Column with a NULL mask) and an
optional ascending uint32 selection vector.  Rows are dicts of Python values
(see rows.py for the JS -> Python mapping).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Any, Iterator, Mapping

import numpy as np

from .engine import Column, Context
from .query import AggregateOp, FilterOp, QueryDescriptor
from .rows import result_to_rows

Row = dict[str, Any]
RowBatch = list[Row]


@dataclass
class ColumnarBatch:
    """ColumnarBatch {columns, rowCount, selection?} (src/operators.ts:57-64)."""
    columns: Mapping[str, Any]
    row_count: int
    selection: np.ndarray | None = None


class Operator:
    def next(self) -> RowBatch | None:
        raise NotImplementedError

    def next_columnar(self) -> ColumnarBatch | None:
        return None

    def close(self) -> None:
        pass


def _values(col) -> tuple[np.ndarray, np.ndarray | None]:
    if isinstance(col, Column):
        return np.asarray(col.values), col.nulls
    return np.asarray(col), None


def materialize_rows(batch: ColumnarBatch) -> RowBatch:
    """materializeRows (src/operators.ts:78-90): NULL cells become None."""
    idx = batch.selection if batch.selection is not None else np.arange(batch.row_count)
    cols = {k: _values(v) for k, v in batch.columns.items()}
    out = []
    for i in idx:
        row = {}
        for name, (vals, nulls) in cols.items():
            if nulls is not None and nulls[i]:
                row[name] = None
            else:
                v = vals[i]
                row[name] = int(v) if vals.dtype.kind in "iu" else float(v)
        out.append(row)
    return out


class ArrayScanOperator(Operator):
    """Yields fixed-size columnar batches of an in-memory table (the shape of
    the reference tests' MockOperator, src/operators-conformance.test.ts:120-139)."""

    def __init__(self, columns: Mapping[str, Any], batch_rows: int = 4096):
        self.columns = columns
        self.batch_rows = batch_rows
        first = next(iter(columns.values()))
        self.n = len(_values(first)[0])
        self.cursor = 0

    def next_columnar(self) -> ColumnarBatch | None:
        if self.cursor >= self.n:
            return None
        a, b = self.cursor, min(self.n, self.cursor + self.batch_rows)
        self.cursor = b
        cols = {}
        for k, v in self.columns.items():
            vals, nulls = _values(v)
            cols[k] = Column(vals[a:b], None if nulls is None else nulls[a:b])
        return ColumnarBatch(cols, b - a)

    def next(self) -> RowBatch | None:
        b = self.next_columnar()
        return None if b is None else materialize_rows(b)


class FilterOperator(Operator):
    """FilterOperator(upstream, filters, filterGroups?) — every batch's
    selection narrowed on the GPU; batches left empty are skipped
    (src/operators.ts:1425-1466)."""

    def __init__(self, upstream: Operator, filters: list[FilterOp], filter_groups: list[list[FilterOp]] | None = None,
                 ctx: Context | None = None, flags: int = 0):
        self.upstream = upstream
        self.filters = list(filters)
        self.filter_groups = filter_groups
        self.ctx = ctx or Context(0)
        self.flags = flags

    def next_columnar(self) -> ColumnarBatch | None:
        q = QueryDescriptor(filters=self.filters, filter_groups=self.filter_groups, flags=self.flags)
        while True:
            batch = self.upstream.next_columnar()
            if batch is None:
                return None
            kept = self.ctx.filter_select(batch.columns, q, batch.selection)
            if kept.size:
                return ColumnarBatch(batch.columns, batch.row_count, kept)

    def next(self) -> RowBatch | None:
        b = self.next_columnar()
        return None if b is None else materialize_rows(b)

    def close(self) -> None:
        self.upstream.close()


class AggregateOperator(Operator):
    """AggregateOperator(upstream, query) — one GPU aggregation over all
    upstream batches in batch order; next() yields every result row once."""

    def __init__(self, upstream: Operator, query: QueryDescriptor, ctx: Context | None = None):
        self.upstream = upstream
        self.query = query
        self.consumed = False
        self.ctx = ctx or getattr(upstream, "ctx", None) or Context(0)

    def _source_and_query(self) -> tuple[Operator, QueryDescriptor]:
        q = replace(self.query, filters=list(self.query.filters), filter_groups=self.query.filter_groups)
        src = self.upstream
        # fuse an upstream GPU filter into the aggregation kernel
        while isinstance(src, FilterOperator):
            q.filters = q.filters + src.filters
            if src.filter_groups:
                if q.filter_groups:
                    # (A or B) and (C or D): distribute into one OR of AND chains
                    q.filter_groups = [g1 + g2 for g1 in q.filter_groups for g2 in src.filter_groups]
                else:
                    q.filter_groups = src.filter_groups
            q.flags |= src.flags
            src = src.upstream
        return src, q

    def next(self) -> RowBatch | None:
        if self.consumed:
            return None
        self.consumed = True
        src, q = self._source_and_query()
        grouped = bool(q.group_by)
        stream = self.ctx.aggregate(q)
        pushed = False
        try:
            while True:
                batch = src.next_columnar()
                if batch is None:
                    break
                stream.push(batch.columns, batch.selection)
                pushed = True
            if not pushed:
                return _empty_result(q)
            return result_to_rows(stream.finish(), grouped)
        finally:
            stream.close()

    def close(self) -> None:
        self.upstream.close()


def _empty_result(q: QueryDescriptor) -> RowBatch:
    """finalizePartialAgg(computePartialAgg([], query)) with no input batch:
    [{}] when grouped, else one row of COUNT 0 / NULL (src/operators.ts:1679)."""
    if q.group_by:
        return [{}]
    return [{a.out_name: (0 if a.fn == "count" else None) for a in (q.aggregates or [])}]


def drain_pipeline(op: Operator) -> RowBatch:
    """drainPipeline (src/operators.ts:3155-3179)."""
    rows: RowBatch = []
    while True:
        b = op.next()
        if b is None:
            return rows
        rows.extend(b)


def iterate(op: Operator) -> Iterator[Row]:
    for r in drain_pipeline(op):
        yield r
