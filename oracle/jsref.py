"""Literal pure-Python restatement of the reference path — TEST INFRASTRUCTURE.

Used only by tests, on small inputs, to pin the C oracle (qm_oracle.c): it
keeps the reference's own data structures — string group keys built with
String(v) joined by NUL (src/types.ts:10-18), a Map in first-seen order, the
PartialAggState fields (src/partial-agg.ts:13-36) — so that the C oracle's
typed-key shortcut can be checked against them.

JS values are modelled as: number -> Python float, bigint -> Python int,
null -> None.
"""
from __future__ import annotations

import math
import re

NULL_SENTINEL = "\x01NULL\x01"  # src/types.ts:2


def js_num_str(x: float) -> str:
    """ECMAScript Number::toString(10) (shortest round-trip digits)."""
    if x != x:
        return "NaN"
    if x == 0:
        return "0"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    if x < 0:
        return "-" + js_num_str(-x)
    s = repr(float(x))
    if "e" in s:
        m, e = s.split("e")
        e = int(e)
    else:
        m, e = s, 0
    ip, fp = (m.split(".") + [""])[:2] if "." in m else (m, "")
    allds = ip + fp
    q = e - len(fp)
    stripped = allds.lstrip("0")
    d = stripped.rstrip("0")
    q += len(stripped) - len(d)
    k = len(d)
    n = q + k
    if k <= n <= 21:
        return d + "0" * (n - k)
    if 0 < n <= 21:
        return d[:n] + "." + d[n:]
    if -6 < n <= 0:
        return "0." + "0" * (-n) + d
    ex = n - 1
    sign = "+" if ex >= 0 else "-"
    if k == 1:
        return d + "e" + sign + str(abs(ex))
    return d[0] + "." + d[1:] + "e" + sign + str(abs(ex))


def js_string(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)  # String(bigint)
    return js_num_str(v)


def group_key_from(vals) -> str:
    """groupKeyFrom (src/types.ts:10-18)."""
    return "\0".join(NULL_SENTINEL if v is None else js_string(v) for v in vals)


def js_number_of(s: str) -> float:
    t = s.strip()
    if t == "NaN":
        return math.nan
    if t in ("Infinity", "+Infinity"):
        return math.inf
    if t == "-Infinity":
        return -math.inf
    try:
        return float(t)
    except ValueError:
        return math.nan


# ---------------------------------------------------------------- predicates
def _trunc_big(x: float) -> int:
    return int(math.trunc(x))


def coerce_compare(a, b):
    """coerceCompare (src/decode.ts:480-485)."""
    if isinstance(a, int) and isinstance(b, float):
        return a, (_trunc_big(b) if math.isfinite(b) else b)
    if isinstance(a, float) and isinstance(b, int):
        return (_trunc_big(a) if math.isfinite(a) else a), b
    return a, b


def _strict_eq(a, b) -> bool:
    if type(a) is not type(b):
        return False
    return a == b


def _lt(a, b) -> bool:  # JS relational, mixed bigint/number compare mathematically
    if isinstance(a, float) and a != a or isinstance(b, float) and b != b:
        return False
    return a < b


def _filter_value(v):
    """A FilterOp value as a JS value: querymode_b200.query.BigInt is a
    bigint, any other Python number is a JS number."""
    from querymode_b200.query import BigInt
    if isinstance(v, (list, tuple)):
        return [_filter_value(x) for x in v]
    if isinstance(v, BigInt):
        return int(v)
    return float(v)


def matches_filter(val, f) -> bool:
    """matchesFilter (src/decode.ts:489-541), numeric ops."""
    op, t = f.op, _filter_value(f.value)
    if op == "eq":
        a, b = coerce_compare(val, t)
        return _strict_eq(a, b)
    if op == "neq":
        a, b = coerce_compare(val, t)
        return not _strict_eq(a, b)
    if op == "gt":
        a, b = coerce_compare(val, t)
        return _lt(b, a)
    if op == "gte":
        a, b = coerce_compare(val, t)
        return _lt(b, a) or (not _nan(a) and not _nan(b) and a == b)
    if op == "lt":
        a, b = coerce_compare(val, t)
        return _lt(a, b)
    if op == "lte":
        a, b = coerce_compare(val, t)
        return _lt(a, b) or (not _nan(a) and not _nan(b) and a == b)
    if op == "between":
        _, lo = coerce_compare(val, t[0])
        a, hi = coerce_compare(val, t[1])
        return _ge(a, lo) and _ge(hi, a)
    if op == "not_between":
        _, lo = coerce_compare(val, t[0])
        a, hi = coerce_compare(val, t[1])
        return _lt(a, lo) or _lt(hi, a)
    return True


def _nan(x) -> bool:
    return isinstance(x, float) and x != x


def _ge(a, b) -> bool:
    if _nan(a) or _nan(b):
        return False
    return a >= b


def row_passes_filters(row: dict, filters, filter_groups=None) -> bool:
    """rowPassesFilters (src/decode.ts:558-578)."""
    for f in filters:
        v = row.get(f.column)
        if f.op == "is_null":
            if v is not None:
                return False
            continue
        if f.op == "is_not_null":
            if v is None:
                return False
            continue
        if v is None:
            return False
        if not matches_filter(v, f):
            return False
    if filter_groups:
        def group_ok(g):
            for f in g:
                v = row.get(f.column)
                if f.op == "is_null":
                    if v is not None:
                        return False
                    continue
                if f.op == "is_not_null":
                    if v is None:
                        return False
                    continue
                if v is None or not matches_filter(v, f):
                    return False
            return True
        return any(group_ok(g) for g in filter_groups)
    return True


# ------------------------------------------------------------- aggregation
class State:
    """PartialAggState (src/partial-agg.ts:13-36), numeric fields."""

    def __init__(self, fn: str, column: str):
        self.fn, self.column = fn, column
        self.sum = 0.0
        self.count = 0
        self.min = math.inf
        self.max = -math.inf
        self.big_sum = None
        self.big_min = None
        self.big_max = None


def update(state: State, value: float) -> None:  # src/partial-agg.ts:63-86
    state.sum += value
    state.count += 1
    if value < state.min:
        state.min = value
    if value > state.max:
        state.max = value


def update_big(state: State, value: int) -> None:  # src/partial-agg.ts:89-95
    state.big_sum = (state.big_sum or 0) + value
    state.count += 1
    if state.big_min is None or value < state.big_min:
        state.big_min = value
    if state.big_max is None or value > state.big_max:
        state.big_max = value


def feed(states, aggregates, get_val) -> None:  # src/partial-agg.ts:141-166
    for i, a in enumerate(aggregates):
        if a.column == "*":
            states[i].count += 1
            continue
        v = get_val(a.column)
        if isinstance(v, float):
            update(states[i], v)
        elif isinstance(v, int):
            update_big(states[i], v)


def merge(t: State, s: State) -> None:  # src/partial-agg.ts:225-267
    t.sum += s.sum
    t.count += s.count
    if s.min < t.min:
        t.min = s.min
    if s.max > t.max:
        t.max = s.max
    if s.big_sum is not None:
        t.big_sum = (t.big_sum or 0) + s.big_sum
        if t.big_min is None or s.big_min < t.big_min:
            t.big_min = s.big_min
        if t.big_max is None or s.big_max > t.big_max:
            t.big_max = s.big_max


def _num_of_big(b: int) -> float:
    return float(b)  # Python int -> float rounds half to even, as Number(bigint)


def big_avg(big_sum: int, num_sum: float, count: int) -> float:  # src/partial-agg.ts:38-44
    q = abs(big_sum) // count * (1 if big_sum >= 0 else -1)  # BigInt '/' truncates
    r = big_sum - q * count                                  # sign of the dividend
    return _num_of_big(q) + (_num_of_big(r) + num_sum) / count


def safe_big(v: float) -> int:  # src/types.ts:21-23
    return int(math.trunc(v)) if math.isfinite(v) else 0


def resolve(s: State):  # src/partial-agg.ts:105-134
    if s.fn == "count":
        return s.count
    if s.count == 0:
        return None
    has_big = s.big_sum is not None
    if s.fn == "sum":
        return s.big_sum + safe_big(s.sum) if has_big else s.sum
    if s.fn == "avg":
        return big_avg(s.big_sum, s.sum, s.count) if has_big else s.sum / s.count
    if s.fn == "min":
        return s.big_min if has_big else s.min
    if s.fn == "max":
        return s.big_max if has_big else s.max
    raise ValueError(s.fn)


def restore_key_part(part: str):  # src/partial-agg.ts:327-344
    if part == NULL_SENTINEL:
        return None
    num = js_number_of(part)
    if part != "" and js_num_str(num) == part:
        return num
    if part != "" and re.fullmatch(r"-?\d+", part):
        return int(part)
    return part


def run(columns: dict, query, batch_rows: int = 0) -> list[dict]:
    """AggregateOperator over batches (src/operators.ts:1656-1681): filter,
    per-batch partial with string keys, merge in batch order, finalize.
    `columns` maps name -> list of JS values (float / int / None)."""
    aggs = query.aggregates or []
    gcols = query.group_by or []
    n = len(next(iter(columns.values()))) if columns else 0
    batch_rows = batch_rows or max(n, 1)
    merged = None  # dict key -> states (insertion ordered) or list of states
    for b0 in range(0, max(n, 0), batch_rows):
        b1 = min(n, b0 + batch_rows)
        rows = [{c: columns[c][r] for c in columns} for r in range(b0, b1)]
        sel = [row for row in rows if row_passes_filters(row, query.filters, query.filter_groups)]
        if not gcols:
            part = [State(a.fn, a.column) for a in aggs]
            for row in sel:
                feed(part, aggs, lambda c, row=row: row.get(c))
        else:
            part = {}
            for row in sel:
                k = group_key_from([row.get(c) for c in gcols])
                st = part.get(k)
                if st is None:
                    st = [State(a.fn, a.column) for a in aggs]
                    part[k] = st
                feed(st, aggs, lambda c, row=row: row.get(c))
        if merged is None:
            merged = part
        elif not gcols:
            for t, s in zip(merged, part):
                merge(t, s)
        else:
            for k, st in part.items():
                if k not in merged:
                    merged[k] = st
                else:
                    for t, s in zip(merged[k], st):
                        merge(t, s)
    if merged is None:
        merged = [State(a.fn, a.column) for a in aggs] if not gcols else {}
    names = [a.alias if a.alias is not None else f"{a.fn}_{a.column}" for a in aggs]
    if not gcols or len(merged) == 0:
        # finalizePartialAgg with no groups: one row of the ungrouped states
        # (an empty GROUP BY therefore yields [{}])
        states = merged if not gcols else []
        return [{names[i]: resolve(s) for i, s in enumerate(states)}]
    out = []
    for k, st in merged.items():
        parts = k.split("\0")
        row = {gcols[i]: restore_key_part(parts[i]) for i in range(len(gcols))}
        for i, s in enumerate(st):
            row[names[i]] = resolve(s)
        out.append(row)
    return out
