"""Seeded synthetic tables and queries of the benchmark workloads.

No public dataset backs this path; these generators produce the shapes,
sizes and value distributions of the workloads the path is measured on
(numpy ``default_rng`` seeded per workload):

* ``orders_1m``      1M rows: status int32 codes {0,1,2}, region int32 0..15,
                     amount float64 lognormal(3, 1);
                     SELECT region, SUM(amount), COUNT(*) WHERE status = 1
                     GROUP BY region.
* ``events_100m``    100M rows: key int64 Zipf(s=1.1) over 65,536 values,
                     qty int32 uniform 1..100, price float64 uniform [0, 1000),
                     ts int64 epoch-ms uniform over one year;
                     WHERE ts in a 30-day window AND qty > 10 GROUP BY key
                     SUM(price), SUM(qty), MIN(price), MAX(price), COUNT(*),
                     AVG(price).
* ``wide_keys_200m`` 200M rows: key int64 uniform over 2^24 values,
                     val float64 normal(0, 1e3), flag int32 Bernoulli(0.01);
                     WHERE flag = 1 AND val > 0 GROUP BY key SUM(val), COUNT(*)
                     (and the same without the filter).
* ``generate_rows``  the operator-conformance formula of the reference
                     (src/operators-conformance.test.ts:98-113) with string
                     columns as int32 dictionary codes.
"""
from __future__ import annotations

import numpy as np

from .query import AggregateOp, FilterOp, QueryDescriptor

YEAR_START_MS = 1_704_067_200_000  # 2024-01-01T00:00:00Z
DAY_MS = 86_400_000


def orders(n: int = 1_000_000, seed: int = 0) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    return {
        "status": rng.integers(0, 3, n, dtype=np.int32),
        "region": rng.integers(0, 16, n, dtype=np.int32),
        "amount": rng.lognormal(3.0, 1.0, n),
    }


def orders_query() -> QueryDescriptor:
    return QueryDescriptor(
        table="orders",
        filters=[FilterOp("status", "eq", 1)],
        group_by=["region"],
        aggregates=[AggregateOp("sum", "amount"), AggregateOp("count", "*")],
    )


def zipf_ranks(rng: np.random.Generator, n: int, n_keys: int, s: float, chunk: int = 1 << 24) -> np.ndarray:
    """Ranks 0..n_keys-1 with P(rank k) proportional to (k+1)^-s, by inverse
    CDF (searchsorted on the normalized cumulative weights)."""
    w = np.arange(1, n_keys + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    out = np.empty(n, dtype=np.int64)
    for i in range(0, n, chunk):
        u = rng.random(min(chunk, n - i))
        out[i:i + len(u)] = np.minimum(np.searchsorted(cdf, u, side="right"), n_keys - 1)
    return out


def events(n: int = 100_000_000, seed: int = 1, n_keys: int = 65_536) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n_keys).astype(np.int64)
    key = perm[zipf_ranks(rng, n, n_keys, 1.1)]
    return {
        "key": key,
        "qty": rng.integers(1, 101, n, dtype=np.int32),
        "price": rng.random(n) * 1000.0,
        "ts": rng.integers(YEAR_START_MS, YEAR_START_MS + 365 * DAY_MS, n, dtype=np.int64),
    }


def events_query(window_start_day: int = 100) -> QueryDescriptor:
    t0 = YEAR_START_MS + window_start_day * DAY_MS
    return QueryDescriptor(
        table="events",
        filters=[FilterOp("ts", "gte", t0), FilterOp("ts", "lt", t0 + 30 * DAY_MS),
                 FilterOp("qty", "gt", 10)],
        group_by=["key"],
        aggregates=[AggregateOp("sum", "price"), AggregateOp("sum", "qty"),
                    AggregateOp("min", "price"), AggregateOp("max", "price"),
                    AggregateOp("count", "*"), AggregateOp("avg", "price")],
    )


def wide_keys(n: int = 200_000_000, seed: int = 2, n_keys: int = 1 << 24) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    return {
        "key": rng.integers(0, n_keys, n, dtype=np.int64),
        "val": rng.normal(0.0, 1e3, n),
        "flag": (rng.random(n) < 0.01).astype(np.int32),
    }


def wide_keys_query(filtered: bool = True) -> QueryDescriptor:
    return QueryDescriptor(
        table="wide",
        filters=[FilterOp("flag", "eq", 1), FilterOp("val", "gt", 0)] if filtered else [],
        group_by=["key"],
        aggregates=[AggregateOp("sum", "val"), AggregateOp("count", "*")],
    )


REGIONS = ["us", "eu", "ap", "sa"]
CATEGORIES = ["A", "B", "C"]


def generate_rows(n: int) -> dict[str, np.ndarray]:
    """The reference's generateRows (src/operators-conformance.test.ts:98-113):
    id = i, region = REGIONS[i % 4] and category = CATEGORIES[i % 3] as int32
    dictionary codes, amount = (i*7+13) % 1000, score = ((i*31) % 997) / 10."""
    i = np.arange(n, dtype=np.int64)
    return {
        "id": i.astype(np.int32),
        "region": (i % 4).astype(np.int32),
        "category": (i % 3).astype(np.int32),
        "amount": ((i * 7 + 13) % 1000).astype(np.int32),
        "score": ((i * 31) % 997).astype(np.float64) / 10.0,
    }


def column_bytes(columns: dict[str, np.ndarray], names) -> int:
    return int(sum(columns[c].nbytes for c in names))


def batch_specs(n_queries: int = 256, seed: int = 3, rows_lo: float = 1e4, rows_hi: float = 5e7,
                card_lo: float = 4, card_hi: float = 1e6) -> list[dict]:
    """Shapes of the batched workload: per query, rows log-uniform in
    [rows_lo, rows_hi], group cardinality log-uniform in [card_lo, card_hi],
    int32 or int64 keys, a float64 lognormal measure and a filter threshold
    giving 1-90% selectivity."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_queries):
        rows = int(np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi))))
        card = max(1, int(np.exp(rng.uniform(np.log(card_lo), np.log(card_hi)))))
        specs.append({
            "rows": rows, "card": card, "key64": bool(rng.random() < 0.5),
            "selectivity": float(rng.uniform(0.01, 0.90)), "seed": int(rng.integers(1 << 31)),
        })
    return specs


def batch_table(spec: dict) -> dict[str, np.ndarray]:
    """One query's table: key (int32 codes 0..card-1, or int64 values drawn
    from `card` random 64-bit values), f (int32 uniform 0..9999), v (float64
    lognormal(0, 1))."""
    rng = np.random.default_rng(spec["seed"])
    n, card = spec["rows"], spec["card"]
    idx = rng.integers(0, card, n)
    if spec["key64"]:
        universe = rng.integers(-(1 << 62), 1 << 62, card, dtype=np.int64)
        key = universe[idx]
    else:
        key = idx.astype(np.int32)
    return {"key": key, "f": rng.integers(0, 10_000, n, dtype=np.int32), "v": rng.lognormal(0.0, 1.0, n)}


def batch_query(spec: dict) -> QueryDescriptor:
    threshold = int(round(spec["selectivity"] * 10_000))
    return QueryDescriptor(
        table="batch", filters=[FilterOp("f", "lt", threshold)], group_by=["key"],
        aggregates=[AggregateOp("sum", "v"), AggregateOp("count", "*"), AggregateOp("min", "v"),
                    AggregateOp("max", "v"), AggregateOp("avg", "v")])
