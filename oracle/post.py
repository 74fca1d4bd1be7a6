"""Test infrastructure: the reference's post-aggregate operators restated,
applied to an oracle Result.

* TopKOperator (src/operators.ts:1716-1841): a heap of LIMIT + OFFSET rows
  under `cmp` (NULL and NaN last, then `<` / `>`, negated for DESC), a row
  replacing the root only when strictly better (`shouldReplace`), rows
  pushed one by one in result order (AggregateOperator has no nextColumnar,
  so the row path `pushRow` runs), extraction by repeated root removal,
  reversed, then `.slice(offset)`.
* InMemorySortOperator (src/operators.ts:1846-1884): Array.prototype.sort
  (stable) with rowComparator (src/types.ts:26-38), then `.slice(offset)`.
* LimitOperator (src/operators.ts:1502-1570): rows [offset, offset + limit).

Values compare as JS values: numbers and bigints mathematically (Python
int / float comparison is exact), -0 equal to 0.
"""
from __future__ import annotations

import math
from functools import cmp_to_key

from querymode_b200.engine import Result


def _sort_values(result: Result, column: str | None):
    cols = {c.name: c for c in result.columns}
    if column not in cols:  # row[col] is undefined for every row
        return [None] * result.n_rows
    return cols[column].pyvalues()


def _last(v) -> bool:
    return v is None or (isinstance(v, float) and math.isnan(v))


def _cmp(av, bv, desc: bool) -> int:
    """TopKOperator.cmp / rowComparator."""
    if _last(av) and _last(bv):
        return 0
    if _last(av):
        return 1
    if _last(bv):
        return -1
    c = -1 if av < bv else (1 if av > bv else 0)
    return -c if desc else c


def topk_order(vals: list, desc: bool, limit: int, offset: int) -> list[int]:
    k = limit + offset
    heap: list[int] = []

    def cmp(a, b):
        return _cmp(vals[a], vals[b], desc)

    def should_replace(r) -> bool:
        nv, rv = vals[r], vals[heap[0]]
        if nv is None:
            return False
        if rv is None:
            return True
        if isinstance(rv, float) and math.isnan(rv):
            return True
        if isinstance(nv, float) and math.isnan(nv):
            return False
        return nv > rv if desc else nv < rv

    def sift_down(arr, i):
        while True:
            t = i
            l, r = 2 * i + 1, 2 * i + 2
            if l < len(arr) and cmp(arr[l], arr[t]) > 0:
                t = l
            if r < len(arr) and cmp(arr[r], arr[t]) > 0:
                t = r
            if t == i:
                break
            arr[i], arr[t] = arr[t], arr[i]
            i = t

    def sift_up(i):
        while i > 0:
            p = (i - 1) >> 1
            if cmp(heap[i], heap[p]) > 0:
                heap[i], heap[p] = heap[p], heap[i]
                i = p
            else:
                break

    for row in range(len(vals)):
        if len(heap) < k:
            heap.append(row)
            sift_up(len(heap) - 1)
        elif len(heap) > 0 and should_replace(row):
            heap[0] = row
            sift_down(heap, 0)
    out = []
    copy = list(heap)
    while copy:
        out.append(copy[0])
        copy[0] = copy[-1]
        copy.pop()
        if copy:
            sift_down(copy, 0)
    out.reverse()
    return out[offset:]


def sort_order(vals: list, desc: bool, offset: int) -> list[int]:
    order = sorted(range(len(vals)), key=cmp_to_key(lambda a, b: _cmp(vals[a], vals[b], desc)))
    return order[offset:]


def limit_order(n: int, limit: int | None, offset: int) -> list[int]:
    end = n if limit is None else min(n, offset + limit)
    return list(range(min(offset, n), end))


def post_aggregate(result: Result, sort_column: str | None, desc: bool, limit: int | None,
                   offset: int = 0) -> Result:
    """The rows the reference's pipeline returns after AggregateOperator
    (src/operators.ts:3116-3128), as a Result with the same columns."""
    if sort_column is not None and limit is not None:
        order = topk_order(_sort_values(result, sort_column), desc, limit, offset)
    elif sort_column is not None:
        order = sort_order(_sort_values(result, sort_column), desc, offset)
    elif limit is not None or offset:
        order = limit_order(result.n_rows, limit, offset)
    else:
        return result
    return result.take(order)
