"""Query descriptors: FilterOp / AggregateOp / QueryDescriptor and their C form.

Mirrors the reference types (src/types.ts:130-145 FilterOp / AggregateOp and
the filter/groupBy/aggregates fields of QueryDescriptor, src/client.ts:1254-1277)
and lowers them to the qm_query structure of include/qm_gpu.h.

A filter value follows JS typing: a Python ``float`` is a JS ``number``; a
Python ``int`` is a JS ``bigint`` when wrapped in :class:`BigInt`, and a plain
``int`` is a ``number`` (JS has no separate integer literal type).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Sequence

from . import _abi as A


class BigInt(int):
    """A JS ``bigint`` filter value (e.g. ``BigInt(5)`` for ``5n``)."""


@dataclass(frozen=True)
class FilterOp:
    """FilterOp {column, op, value} (src/types.ts:130-134)."""
    column: str
    op: str
    value: Any = None


@dataclass(frozen=True)
class AggregateOp:
    """AggregateOp {fn, column, alias} (src/types.ts:137-145)."""
    fn: str
    column: str
    alias: str | None = None

    @property
    def out_name(self) -> str:
        # aliasFor, src/partial-agg.ts:136-138
        return self.alias if self.alias is not None else f"{self.fn}_{self.column}"


@dataclass
class QueryDescriptor:
    """The part of QueryDescriptor the filter -> GROUP BY path reads."""
    table: str = ""
    filters: list[FilterOp] = field(default_factory=list)
    filter_groups: list[list[FilterOp]] | None = None
    group_by: list[str] | None = None
    aggregates: list[AggregateOp] | None = None
    flags: int = 0
    # post-aggregate ORDER BY / LIMIT / OFFSET (QueryDescriptor.sortColumn,
    # sortDirection, limit, offset)
    sort_column: str | None = None
    sort_desc: bool = False
    limit: int | None = None
    offset: int = 0


def _value(v: Any) -> A.QmValue:
    out = A.QmValue()
    if isinstance(v, BigInt):
        if not -(1 << 63) <= int(v) < (1 << 63):
            raise ValueError("bigint filter value outside int64")
        out.kind = A.QM_VAL_BIGINT
        out.big = int(v)
    elif isinstance(v, (int, float)) and not isinstance(v, bool):
        out.kind = A.QM_VAL_NUMBER
        out.num = float(v)
    else:
        raise TypeError(f"filter value {v!r} is not numeric (the GPU path filters numbers)")
    return out


def _filter(f: FilterOp, keep: list) -> A.QmFilter:
    if f.op not in A.OP_CODES:
        raise NotImplementedError(f"filter op {f.op!r} is not on the GPU path")
    out = A.QmFilter()
    name = f.column.encode()
    keep.append(name)
    out.column = name
    out.op = A.OP_CODES[f.op]
    if f.op in ("between", "not_between"):
        if not isinstance(f.value, (list, tuple)) or len(f.value) != 2:
            raise ValueError(f"{f.op} needs [low, high]")
        out.value = _value(f.value[0])
        out.value2 = _value(f.value[1])
    elif f.op in ("is_null", "is_not_null"):
        pass
    else:
        out.value = _value(f.value)
    return out


class CQuery:
    """A qm_query plus every buffer it points into (kept alive together)."""

    def __init__(self, q: QueryDescriptor):
        keep: list = []
        fl = [_filter(f, keep) for f in q.filters]
        self.filters = (A.QmFilter * max(1, len(fl)))(*fl)
        groups = q.filter_groups or []
        flat = [_filter(f, keep) for g in groups for f in g]
        self.or_filters = (A.QmFilter * max(1, len(flat)))(*flat)
        self.or_sizes = (C.c_int32 * max(1, len(groups)))(*[len(g) for g in groups])
        gb = [c.encode() for c in (q.group_by or [])]
        keep.extend(gb)
        self.group_by = (C.c_char_p * max(1, len(gb)))(*gb)
        aggs = []
        for a in q.aggregates or []:
            if a.fn not in A.AGG_CODES:
                raise NotImplementedError(f"aggregate {a.fn!r} is not on the GPU path")
            ca = A.QmAggregate()
            ca.fn = A.AGG_CODES[a.fn]
            col = a.column.encode()
            keep.append(col)
            ca.column = col
            if a.alias is not None:
                al = a.alias.encode()
                keep.append(al)
                ca.alias = al
            aggs.append(ca)
        self.aggregates = (A.QmAggregate * max(1, len(aggs)))(*aggs)
        self._keep = keep
        s = A.QmQuery()
        s.filters = self.filters
        s.n_filters = len(fl)
        s.n_or_groups = len(groups)
        s.or_group_sizes = self.or_sizes
        s.or_filters = self.or_filters
        s.group_by = self.group_by
        s.n_group_by = len(gb)
        s.n_aggregates = len(aggs)
        s.aggregates = self.aggregates
        s.flags = q.flags
        if q.sort_column is not None:
            oc = q.sort_column.encode()
            keep.append(oc)
            s.order_by = oc
            s.order_desc = 1 if q.sort_desc else 0
        if q.limit is not None:
            s.has_limit = 1
            s.limit = int(q.limit)
        s.offset = int(q.offset or 0)
        self.struct = s

    @property
    def ref(self):
        return C.byref(self.struct)


def flatten_filters(filters: Sequence[FilterOp] | None) -> list[FilterOp]:
    return list(filters or [])
