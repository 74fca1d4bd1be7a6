"""Autotuner for the batched launch.

Times a batch run as per-query specialised launches (mode 1) and as
per-class persistent kernels (mode 0) under a grid of launch shapes — tiles of 256 rows
per work chunk, block-local table budget (KiB of shared memory; 0 places
every group table in global memory only) and resident blocks per SM — each
at several wave counts (the batch cut into waves whose result copies overlap
the later waves), and keeps the fastest.  Choices persist in a JSON tuning table keyed by a workload
signature (GPU, query count, total-row bucket), so a later batch of the same
shape starts from the stored choice.
"""
from __future__ import annotations

import json
import math
import os
import time

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
DEFAULT_GRID = {
    "chunk_tiles": [128, 512, 2048],
    "local_kb": [0, 24, 40, 96, 160],
    "blocks_per_sm": [0, 1],
    "waves": [1, 4, 8, 16],
}


def signature(batch, device_name: str = "") -> str:
    st = batch.stats()
    bucket = int(math.log2(max(st["rows"], 1)))
    return f"{device_name}|n={batch.n}|rows~2^{bucket}"


def _time(batch, reps: int) -> float:
    batch.run()  # capture / warm
    best = float("inf")
    for _ in range(reps):
        batch.run()
        best = min(best, batch.stats()["device_ms"])
    return best


def tune_batch(batch, grid: dict | None = None, reps: int = 2, table_path: str | None = DEFAULT_TABLE,
               device_name: str = "") -> dict:
    """Search the grid, apply the fastest shape to `batch`, record it in the
    tuning table and return {"choice", "ms", "trials"}."""
    grid = {**DEFAULT_GRID, **(grid or {})}
    trials = []
    t0 = time.perf_counter()
    # per-query launches (the chunk / local-table knobs do not apply)
    batch.set_mode(1)
    for wv in grid["waves"]:
        batch.set_waves(wv)
        trials.append({"mode": 1, "chunk_tiles": 0, "local_kb": 0, "blocks_per_sm": 0, "waves": wv,
                       "ms": _time(batch, reps)})
    # the persistent kernels' shapes at the best wave count of mode 1
    wv = min(trials, key=lambda t: t["ms"])["waves"]
    batch.set_waves(wv)
    batch.set_mode(0)
    for ct in grid["chunk_tiles"]:
        for lk in grid["local_kb"]:
            for bps in grid["blocks_per_sm"]:
                batch.set_tuning(ct, lk, bps)
                ms = _time(batch, reps)
                trials.append({"mode": 0, "chunk_tiles": ct, "local_kb": lk, "blocks_per_sm": bps, "waves": wv,
                               "ms": ms})
    best = min(trials, key=lambda t: t["ms"])
    apply_choice(batch, best)
    out = {"choice": {k: best[k] for k in ("mode", "chunk_tiles", "local_kb", "blocks_per_sm", "waves")},
           "ms": best["ms"],
           "trials": trials, "search_s": time.perf_counter() - t0}
    if table_path:
        save_choice(table_path, signature(batch, device_name), out["choice"], best["ms"])
    return out


def apply_choice(batch, choice: dict) -> None:
    mode = choice.get("mode", 0)
    batch.set_mode(mode)
    if mode == 0:
        batch.set_tuning(choice["chunk_tiles"], choice["local_kb"], choice["blocks_per_sm"])
    batch.set_waves(choice.get("waves", 0))


def load_table(path: str = DEFAULT_TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save_choice(path: str, sig: str, choice: dict, ms: float) -> None:
    table = load_table(path)
    table[sig] = {**choice, "ms": ms}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply_stored(batch, path: str = DEFAULT_TABLE, device_name: str = "") -> dict | None:
    """Apply the stored choice for this batch's signature, if any."""
    entry = load_table(path).get(signature(batch, device_name))
    if entry:
        apply_choice(batch, entry)
    return entry
