#!/usr/bin/env python
"""Filter -> GROUP BY scan throughput on B200.

One step = one filter -> GROUP BY query over one synthetic table resident in
HBM: the events_100m workload (100M rows: key int64 Zipf(1.1) over 65,536
values, qty int32, price float64, ts int64; WHERE ts in a 30-day window AND
qty > 10; GROUP BY key SUM(price), SUM(qty), MIN(price), MAX(price),
COUNT(*), AVG(price)), run through the C ABI (qm_query_run) including the
result's copy back to the host.

  value    scanned GB/s: algorithmic bytes (rows x 28 B of referenced
           columns) of all ranks / the slowest rank's device time
  e2e      the same metric through the C ABI with HOST inputs: table upload
           from pinned memory, query, result download, every step
  roofline the fused scan kernel: algorithmic bytes per launch / its average
           CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (a C restatement of the reference's JS path)
           on a bounded sample, rank 0, N=1 only

Multi-GPU: one process per GPU under torchrun; every rank scans its own
100M-row table (weak scaling, no collective on the data path).

--impl reference times the reference's algorithm on the host cores instead
(its TypeScript/WASM engine cannot run on this image; the oracle port of it
is what runs), over a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "filter+group-by scan GB/s vs HBM peak; served queries/s and p50/p99 latency"
WORKLOAD = "events_100m"
BYTES_PER_ROW = 28  # ts int64 + qty int32 + key int64 + price float64


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--rows", type=int, default=100_000_000)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-sample-rows", type=int, default=8_000_000)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-ingest", action="store_true")
    p.add_argument("--no-parity", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the orders_1m / wide_keys_200m lines")
    p.add_argument("--config-steps", type=int, default=20)
    p.add_argument("--configs", default="orders,filtered,unfiltered",
                   help="which of the orders_1m / wide_keys filtered / unfiltered lines to run")
    p.add_argument("--wide-rows", type=int, default=200_000_000, help="rows of the wide_keys lines")
    p.add_argument("--ingest-reps", type=int, default=3)
    p.add_argument("--serve-queries", type=int, default=1600, help="requests per offered load and repeat")
    p.add_argument("--serve-repeats", type=int, default=3)
    p.add_argument("--serve-burst", type=int, default=800, help="requests of the closed capacity burst")
    p.add_argument("--serve-plain", type=int, default=400, help="requests of the plain per-query comparison")
    p.add_argument("--serve-lanes", type=int, default=8)
    p.add_argument("--serve-max-rows", type=int, default=1 << 29, help="rows a serving batch may scan")
    p.add_argument("--serve-max-groups", type=int, default=1 << 22,
                   help="a request planned at more groups runs alone (heavy)")
    p.add_argument("--serve-loads", default="0.25,0.5,0.75,0.9", help="offered loads as fractions of capacity")
    p.add_argument("--batch-queries", type=int, default=256)
    p.add_argument("--batch-reps", type=int, default=3)
    p.add_argument("--batch-choice", default="",
                   help="mode,chunk_tiles,local_kb,blocks_per_sm,waves for the batch instead of the autotuner's search")
    return p.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(rows: int):
    """DRAM bytes per scan launch over `rows` rows, from the per-row traffic
    in the committed ncu summary (traffic grows in proportion to rows)."""
    path = os.path.join(ROOT, "profiles", "qm_scan_kernel_events_100m.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_row:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) * rows if m else None


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML from a
    thread during the timed region (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.handle = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _run(self):
        import pynvml
        while not self.stop.is_set():
            try:
                mhz = pynvml.nvmlDeviceGetClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
                reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        try:
            import pynvml
            self.handle = self._handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.handle = None
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.handle is not None:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return None
        reasons = sorted(name for name, bit in self.REASONS.items() if any(r & bit for _, r in self.samples))
        return {"sm_mhz": float(np.median([m for m, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "nvml"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(cols, q, sample_rows: int):
    """The CPU oracle over the first `sample_rows` rows, on all host threads
    (and one thread, reported alongside)."""
    import oracle
    sub = {k: np.ascontiguousarray(v[:sample_rows]) for k, v in cols.items()}
    n = len(next(iter(sub.values())))
    threads = os.cpu_count() or 1
    oracle.run(sub, q, batch_rows=1 << 20, threads=threads)  # warm
    t0 = time.perf_counter()
    oracle.run(sub, q, batch_rows=1 << 20, threads=threads)
    t_mt = time.perf_counter() - t0
    n1 = min(n, 2_000_000)
    sub1 = {k: v[:n1] for k, v in sub.items()}
    t0 = time.perf_counter()
    oracle.run(sub1, q, batch_rows=0, threads=1)
    t_1 = time.perf_counter() - t0
    return {
        "value": n * BYTES_PER_ROW / t_mt / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
        "sample": f"first {n:,} rows of {WORKLOAD} ({n * BYTES_PER_ROW / 1e9:.2f} GB), oracle on {threads} threads",
        "single_thread_gbs": n1 * BYTES_PER_ROW / t_1 / 1e9,
    }


def check_parity(res, cols, q) -> dict:
    """The last timed step's result against the oracle's one-batch result over
    the same table (the checker, run after the timed region)."""
    import oracle
    from tests.helpers import assert_same
    t0 = time.perf_counter()
    ref = oracle.run_full(cols, q)
    try:
        assert_same(res, ref)
        ok, why = True, ""
    except AssertionError as e:
        ok, why = False, str(e)[:300]
    return {"ok": ok, "groups": int(ref.n_rows), "oracle": "one batch, key-partitioned host threads",
            "threads": os.cpu_count() or 1, "seconds": round(time.perf_counter() - t0, 2), "detail": why}


def run_config(ctx, stream, name: str, cols: dict, q, bytes_per_row: int, steps: int, warmup: int,
               cpu_rows: int, note: str, args=None) -> dict:
    """One more of the measured workloads, on one GPU: device-resident table
    (`value`: algorithmic bytes / CUDA-event time per query, result in host
    memory), the scan kernel's roofline, the same query end to end from
    pinned host columns (`e2e`), the oracle on a bounded sample of the host
    cores (`cpu_baseline`) and the benched result against the oracle."""
    import torch

    import oracle
    from querymode_b200.query import CQuery
    n = len(next(iter(cols.values())))
    cq = CQuery(q)
    peak, peak_kind = load_peaks()
    with torch.cuda.stream(stream):
        t = ctx.table(cols)
        for _ in range(max(3, warmup)):
            res = t.run(cq)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        scan, launches = [], 0
        e0.record(stream)
        for _ in range(steps):
            res = t.run(cq)
            scan.append(res.stats.scan_ms)
            launches += res.stats.launches
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        t.close()
    e2e = None
    if not (args and args.no_e2e):
        e2e = run_config_e2e(ctx, stream, cols, cq, n * bytes_per_row)
    qbytes = n * bytes_per_row
    scan_ms = float(np.mean(scan))
    achieved = qbytes / (scan_ms / 1e3) / 1e9
    cpu = None
    if not (args and args.no_cpu):
        sub = {k: np.ascontiguousarray(v[:cpu_rows]) for k, v in cols.items()}
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.run_full(sub, q, threads=threads)
        cpu_s = time.perf_counter() - t0
        sub_rows = len(next(iter(sub.values())))
        cpu = {"value": sub_rows * bytes_per_row / cpu_s / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"first {sub_rows:,} rows, oracle one batch on {threads} threads"}
    parity = None if (args and args.no_parity) else check_parity(res, cols, q)
    return {
        "workload": name, "rows": n, "bytes_per_row": bytes_per_row, "groups": int(res.n_rows),
        "rows_selected": int(res.stats.rows_selected), "steps": steps, "warmup": max(3, warmup),
        "ms_per_query": ms, "value": qbytes / (ms / 1e3) / 1e9, "unit": "GB/s", "rows_per_s": n / (ms / 1e3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "qm_scan_kernel", "kernel_ms": scan_ms},
        "e2e": e2e, "cpu_baseline": cpu,
        "parity": None if parity is None else parity["ok"], "parity_check": parity, "gpu_launches": launches,
        "note": note,
    }


def run_config_e2e(ctx, stream, cols: dict, cq, qbytes: int) -> dict:
    """The query end to end from pinned host columns: upload, query, result
    download, every step, CUDA events on the context's stream."""
    import torch
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        pinned = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in cols.items()}
        h2d = sum(v.nbytes for v in pinned.values())
        tt = ctx.table(pinned)
        r = tt.run(cq)
        tt.close()
        d2h = sum(c.values.nbytes for c in r.columns)
        torch.cuda.synchronize()
        e0.record(stream)
        e2e_steps = 3
        for _ in range(e2e_steps):
            tt = ctx.table(pinned)
            tt.run(cq)
            tt.close()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e2e_steps
        del pinned
    return {"value": qbytes / (e2e_ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms, "steps": e2e_steps}


def run_configs(ctx, stream, args) -> dict:
    """orders_1m (16 groups, launch-bound) and wide_keys_200m filtered /
    unfiltered (16.7M groups, hash table beyond L2)."""
    from querymode_b200 import datagen
    out = {}
    which = set(args.configs.split(","))
    if "orders" in which:
        orders = datagen.orders(1_000_000, seed=0)
        out["orders_1m"] = run_config(ctx, stream, "orders_1m", orders, datagen.orders_query(), 16,
                                      max(args.config_steps, 50), args.warmup, 1_000_000,
                                      "status = 1 GROUP BY region SUM(amount), COUNT(*); 16 groups; launch- and "
                                      "sync-bound (16 MB per query)", args)
        del orders
    if not which & {"filtered", "unfiltered"}:
        return out
    wide = datagen.wide_keys(args.wide_rows, seed=2, n_keys=1 << 24)
    wname = "wide_keys_200m" if args.wide_rows == 200_000_000 else f"wide_keys_{args.wide_rows}"
    if "filtered" in which:
        out[f"{wname}_filtered"] = run_config(
            ctx, stream, f"{wname}_filtered", wide, datagen.wide_keys_query(True), 20, args.config_steps, args.warmup,
            20_000_000, "flag = 1 AND val > 0 (~0.5 %) GROUP BY key SUM(val), COUNT(*); key int64 over 2^24 values",
            args)
    if "unfiltered" in which:
        out[f"{wname}_unfiltered"] = run_config(
            ctx, stream, f"{wname}_unfiltered", wide, datagen.wide_keys_query(False), 16,
            max(3, args.config_steps // 4), args.warmup, 20_000_000,
            "no filter, GROUP BY key SUM(val), COUNT(*): 16.7M groups, result 0.4 GB to the host", args)
    return out


def batch_tables_on_device(specs, device: int):
    """The batched workload's tables generated on the device (seeded torch
    generator per query), read in place by the library."""
    import torch
    g = torch.Generator(device=f"cuda:{device}")
    out = []
    for s in specs:
        g.manual_seed(s["seed"])
        n, card = s["rows"], s["card"]
        idx = torch.randint(0, card, (n,), device=f"cuda:{device}", generator=g)
        if s["key64"]:
            universe = torch.randint(-(1 << 62), 1 << 62, (card,), dtype=torch.int64, device=f"cuda:{device}",
                                     generator=g)
            key = universe[idx]
        else:
            key = idx.to(torch.int32)
        del idx
        f = torch.randint(0, 10_000, (n,), dtype=torch.int32, device=f"cuda:{device}", generator=g)
        v = torch.empty(n, dtype=torch.float64, device=f"cuda:{device}").log_normal_(0.0, 1.0, generator=g)
        out.append({"key": key, "f": f, "v": v})
    return out


def run_batched(ctx, stream, local: int, args) -> dict:
    """256 filter -> GROUP BY queries of uneven sizes as one batched run
    (autotuned between per-query launches and per-class persistent kernels,
    cut into waves, each wave graph-replayed) against the same queries as
    sequential per-query runs; both end with every result in host memory."""
    import torch

    from querymode_b200 import autotune, datagen
    from querymode_b200.query import CQuery
    specs = datagen.batch_specs(args.batch_queries, seed=3)
    dev_tables = batch_tables_on_device(specs, local)
    tables = [ctx.table(t) for t in dev_tables]
    cqs = [CQuery(datagen.batch_query(s)) for s in specs]
    batch = ctx.batch(tables, cqs)
    if args.batch_choice:
        keys = ("mode", "chunk_tiles", "local_kb", "blocks_per_sm", "waves")
        choice = dict(zip(keys, (int(x) for x in args.batch_choice.split(","))))
        autotune.apply_choice(batch, choice)
        tuned = {"choice": choice, "search_s": 0.0, "trials": []}
    else:
        tuned = autotune.tune_batch(batch, reps=1, device_name=torch.cuda.get_device_name(local))

    def timed(fn, reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, (time.perf_counter() - t0) * 1e3 / reps

    def plain():
        for t, q in zip(tables, cqs):
            t.run(q)

    with torch.cuda.stream(stream):
        plain_ms, plain_wall = timed(plain, max(1, args.batch_reps))
        batch_ms, batch_wall = timed(batch.run, max(3, args.batch_reps))
    st = batch.stats()
    n = len(specs)
    out = {
        "queries": n, "rows": st["rows"], "bytes": st["bytes"], "chunks": st["chunks"],
        "plain_ms": plain_ms, "batched_ms": batch_ms, "plain_qps": n / (plain_ms / 1e3),
        "batched_qps": n / (batch_ms / 1e3), "speedup": plain_ms / batch_ms,
        "batched_scan_gbs": st["bytes"] / (st["device_ms"] / 1e3) / 1e9,
        "batched_scan_frac": st["bytes"] / (st["device_ms"] / 1e3) / 1e9 / load_peaks()[0],
        "plain_wall_ms": plain_wall, "batched_wall_ms": batch_wall,
        "autotune": {"choice": tuned["choice"], "search_s": round(tuned["search_s"], 2),
                     "trials": len(tuned["trials"])},
        "workload": "256 queries, rows log-uniform 1e4..5e7, cardinality log-uniform 4..1e6, int32/int64 keys, "
                    "1-90% selectivity (seed 3)",
    }
    batch.close()
    for t in tables:
        t.close()
    del dev_tables
    torch.cuda.empty_cache()
    return out


def serving_tables(device: int) -> dict:
    """The serving mix's eight resident tables, generated on the device
    (seeded): the orders / events / wide-keys shapes at 1M-200M rows, each
    with payload columns the mix's queries do not read (as a table holds more
    columns than one query touches), ~59 GB in all."""
    import torch
    dev = f"cuda:{device}"
    g = torch.Generator(device=dev)

    def payload(n, spec):
        out = {}
        for name, dt in spec:
            if dt == "i64":
                out[name] = torch.randint(0, 1 << 40, (n,), dtype=torch.int64, device=dev, generator=g)
            elif dt == "i32":
                out[name] = torch.randint(0, 1 << 20, (n,), dtype=torch.int32, device=dev, generator=g)
            else:
                out[name] = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
        return out

    def orders(n, seed, extra=()):
        g.manual_seed(seed)
        cols = {"status": torch.randint(0, 3, (n,), dtype=torch.int32, device=dev, generator=g),
                "region": torch.randint(0, 16, (n,), dtype=torch.int32, device=dev, generator=g),
                "amount": torch.empty(n, dtype=torch.float64, device=dev).log_normal_(3.0, 1.0, generator=g)}
        cols.update(payload(n, extra))
        return cols

    def events(n, seed, n_keys=65_536, extra=()):
        g.manual_seed(seed)
        w = torch.arange(1, n_keys + 1, dtype=torch.float64, device=dev) ** -1.1
        cdf = torch.cumsum(w, 0)
        cdf /= cdf[-1].clone()
        perm = torch.randperm(n_keys, device=dev, generator=g)
        key = torch.empty(n, dtype=torch.int64, device=dev)
        for i in range(0, n, 1 << 25):
            u = torch.rand(min(1 << 25, n - i), dtype=torch.float64, device=dev, generator=g)
            key[i:i + len(u)] = perm[torch.searchsorted(cdf, u, right=True).clamp_(max=n_keys - 1)]
        cols = {"key": key,
                "qty": torch.randint(1, 101, (n,), dtype=torch.int32, device=dev, generator=g),
                "price": torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 1000.0,
                "ts": torch.randint(datagen_year_start(), datagen_year_start() + 365 * 86_400_000, (n,),
                                    dtype=torch.int64, device=dev, generator=g)}
        cols.update(payload(n, extra))
        return cols

    def wide(n, seed, n_keys=1 << 24, extra=()):
        g.manual_seed(seed)
        cols = {"key": torch.randint(0, n_keys, (n,), dtype=torch.int64, device=dev, generator=g),
                "val": torch.randn(n, dtype=torch.float64, device=dev, generator=g) * 1e3,
                "flag": (torch.rand(n, device=dev, generator=g) < 0.01).to(torch.int32)}
        cols.update(payload(n, extra))
        return cols

    ord_x = (("customer", "i64"), ("discount", "f64"), ("channel", "i32"), ("ship_ts", "i64"))
    ev_x = (("user", "i64"), ("session", "i64"), ("amount", "f64"), ("referrer", "i64"))
    wide_x = (("aux", "i64"), ("w", "f64"), ("z", "f64"))
    return {"orders_1m": ("orders", orders(1_000_000, 40)),
            "orders_200m": ("orders", orders(200_000_000, 41, ord_x)),
            "events_100m": ("events", events(100_000_000, 42, extra=ev_x)),
            "events_200m_a": ("events", events(200_000_000, 43, extra=ev_x)),
            "events_200m_b": ("events", events(200_000_000, 44, extra=ev_x)),
            "wide_50m": ("wide", wide(50_000_000, 45, extra=wide_x)),
            "wide_200m_a": ("wide", wide(200_000_000, 46, extra=wide_x)),
            "wide_200m_b": ("wide", wide(200_000_000, 47, extra=wide_x))}


def datagen_year_start() -> int:
    from querymode_b200 import datagen
    return datagen.YEAR_START_MS


def run_serving(local: int, args) -> dict:
    """Poisson arrivals of single requests mixing the orders / events /
    wide-keys queries over 8 resident tables (~59 GB), served by the native
    multi-lane continuous-batching server under a 150 GB HBM budget; latency
    = submit -> result in host memory, per offered load, each load repeated;
    against the same request mix run as plain per-query launches."""
    import threading

    import torch

    from querymode_b200 import datagen
    from querymode_b200.engine import Context
    from querymode_b200.query import AggregateOp, CQuery, FilterOp, QueryDescriptor

    rng = np.random.default_rng(4)
    tabs = serving_tables(local)
    torch.cuda.synchronize()
    table_bytes = sum(t.numel() * t.element_size() for _, cols in tabs.values() for t in cols.values())
    sctx = Context(local)
    handles = {name: (kind, sctx.table(cols)) for name, (kind, cols) in tabs.items()}

    # request templates per table kind (query objects built once)
    events_q = [CQuery(datagen.events_query(window_start_day=int(d))) for d in rng.integers(0, 330, 48)]
    orders_q = [CQuery(QueryDescriptor(filters=[FilterOp("status", "eq", s)], group_by=["region"],
                                       aggregates=[AggregateOp("sum", "amount"), AggregateOp("count", "*")]))
                for s in range(3)]
    wide_q = [CQuery(datagen.wide_keys_query(True)),
              CQuery(QueryDescriptor(filters=[FilterOp("flag", "eq", 1)], group_by=["key"],
                                     aggregates=[AggregateOp("max", "val"), AggregateOp("count", "*")]))]
    wide_full = CQuery(datagen.wide_keys_query(False))
    names = list(handles)

    def draw(r):
        name = names[int(r.integers(len(names)))]
        kind, t = handles[name]
        if kind == "orders":
            return t, orders_q[int(r.integers(3))]
        if kind == "events":
            return t, events_q[int(r.integers(len(events_q)))]
        if r.random() < 0.01:  # the unfiltered 16M-group aggregate, rarely
            return t, wide_full
        return t, wide_q[int(r.integers(2))]

    # a batch scans at most --serve-max-rows rows; requests planned at more
    # than --serve-max-groups groups (the 16M-group aggregate) run alone
    # (heavy); the last of the lanes takes light requests only
    srv = sctx.server(hbm_budget_bytes=150_000_000_000, max_batch=64, max_wait_us=0,
                      max_batch_rows=args.serve_max_rows, lanes=args.serve_lanes,
                      max_batch_groups=args.serve_max_groups)
    try:
        # warm-up: every table and query kind on every lane (column statistics are cached)
        for _ in range(args.serve_lanes):
            warm = []
            for name, (kind, t) in handles.items():
                qs = orders_q if kind == "orders" else (events_q[:2] if kind == "events" else wide_q + [wide_full])
                warm += [srv.submit(t, q) for q in qs]
            for tk in warm:
                srv.wait(tk)

        def serve(reqs, rate):
            """Submit reqs at Poisson arrivals of `rate` per second (all at
            once if rate is None); returns (latencies us, batch sizes, span s)."""
            tickets = [None] * len(reqs)
            lat, bs = [0.0] * len(reqs), [0] * len(reqs)
            gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
            done_at = [0.0]

            def collect():
                for i in range(len(reqs)):
                    while tickets[i] is None:
                        time.sleep(0)
                    _, tm = srv.wait(tickets[i])
                    lat[i], bs[i] = tm["total_us"], tm["batch_size"]
                done_at[0] = time.perf_counter()

            th = threading.Thread(target=collect)
            th.start()
            t0 = time.perf_counter()
            due = t0
            for i, (t, q) in enumerate(reqs):
                due += gaps[i]
                rem = due - time.perf_counter()
                if rem > 0.002:
                    time.sleep(rem - 0.001)
                while time.perf_counter() < due:
                    pass
                tickets[i] = srv.submit(t, q)
            th.join()
            return np.array(lat), np.array(bs), done_at[0] - t0

        # capacity: closed bursts of requests.  The first burst grows the
        # lanes' buffers and the pinned result pool to the mix's working set
        # (reported as the cold capacity); the last one is the steady state.
        burst = [draw(rng) for _ in range(args.serve_burst)]
        _, _, span = serve(burst, None)
        cold_capacity = len(burst) / span
        serve(burst, None)
        _, bsz, span = serve(burst, None)
        capacity = len(burst) / span
        loads = []
        served = 0
        for frac in [float(x) for x in args.serve_loads.split(",")]:
            reps = []
            for _ in range(args.serve_repeats):
                reqs = [draw(rng) for _ in range(args.serve_queries)]
                lat, bsz, span = serve(reqs, capacity * frac)
                served += len(reqs)
                reps.append({"achieved_qps": round(len(reqs) / span, 1),
                             "p50_ms": round(float(np.percentile(lat, 50)) / 1e3, 3),
                             "p95_ms": round(float(np.percentile(lat, 95)) / 1e3, 3),
                             "p99_ms": round(float(np.percentile(lat, 99)) / 1e3, 3),
                             "mean_batch": round(float(bsz.mean()), 2)})
            med = lambda k: round(float(np.median([r[k] for r in reps])), 3)
            loads.append({"offered_qps": round(capacity * frac, 1), "achieved_qps": med("achieved_qps"),
                          "p50_ms": med("p50_ms"), "p95_ms": med("p95_ms"), "p99_ms": med("p99_ms"),
                          "mean_batch": med("mean_batch"), "p99_ms_repeats": [r["p99_ms"] for r in reps],
                          "repeats": reps})
        st = srv.stats()
    finally:
        srv.close()
    # the same request mix as plain per-query launches (Table.run, result
    # in host memory), closed loop
    plain_reqs = [draw(rng) for _ in range(args.serve_plain)]
    for t, q in plain_reqs:  # one untimed pass: buffers and pinned pool at the mix's size
        t.run(q)
    t0 = time.perf_counter()
    for t, q in plain_reqs:
        t.run(q)
    plain_qps = len(plain_reqs) / (time.perf_counter() - t0)
    sctx.close()
    del tabs, handles
    torch.cuda.empty_cache()
    return {"tables": 8, "table_gb": round(table_bytes / 1e9, 2), "hbm_budget_gb": 150, "lanes": st["lanes"],
            "max_batch_rows": args.serve_max_rows, "max_batch_groups": args.serve_max_groups,
            "capacity_qps": round(capacity, 1), "cold_capacity_qps": round(cold_capacity, 1),
            "plain_qps": round(plain_qps, 1),
            "served_vs_plain": round(capacity / plain_qps, 2),
            "queries": served + len(burst), "queries_per_load": args.serve_queries * args.serve_repeats,
            "repeats": args.serve_repeats, "loads": loads,
            "server": {k: st[k] for k in ("completed", "failed", "refused", "batches", "peak_working_bytes",
                                          "peak_in_flight", "heavy")},
            "mix": "uniform over 8 tables (orders 1M/200M, events 100M/200M/200M, wide 50M/200M/200M); "
                   "orders: status filter by region; events: 30-day window + qty, 48 windows; wide: flag (+val) "
                   "filters, 1% unfiltered 16M-group; Poisson arrivals (seed 4); plain: the same mix, one "
                   "Table.run after another"}


def run_ingest(ctx, cols: dict, args) -> dict:
    """Scan pages in host memory -> a device table (qm_table_from_pages): the
    events columns as 10,000-row pages (the page size of the reference's
    benchmark data), each column's pages back to back in one host buffer
    with a page table (offset, length, rowCount, nullCount), as a reader
    holds a column's byte range; key, qty and ts plain, price with a
    validity bitmap (1 % NULL) and its non-NULL values packed behind it.
    Timed end to end (staging through pinned buffers, H2D, decode kernels)
    by the host clock around the synchronous call."""
    from querymode_b200 import _abi as A
    from querymode_b200.engine import PageTable

    rows_per_page = 10_000
    n = len(next(iter(cols.values())))
    rng = np.random.default_rng(5)
    price_null = rng.random(n) < 0.01
    types = {"key": A.QM_I64, "qty": A.QM_I32, "price": A.QM_F64, "ts": A.QM_I64}
    starts = np.arange(0, n, rows_per_page, dtype=np.int64)
    counts = np.minimum(rows_per_page, n - starts)
    spec = []
    page_bytes = 0
    for name, qd in types.items():
        v = cols[name]
        if name == "price":
            parts, lens, nulls = [], [], []
            for a, c in zip(starts, counts):
                m = price_null[a:a + c]
                parts += [np.packbits(~m, bitorder="little"), v[a:a + c][~m].view(np.uint8)]
                lens.append(parts[-2].nbytes + parts[-1].nbytes)
                nulls.append(int(m.sum()))
            buf = np.concatenate(parts)
            lens = np.array(lens, dtype=np.int64)
            pt = PageTable(buf, np.concatenate([[0], np.cumsum(lens)[:-1]]), lens, counts, np.array(nulls))
        else:
            buf = v.view(np.uint8)
            pt = PageTable(buf, starts * v.itemsize, counts * v.itemsize, counts)
        page_bytes += buf.nbytes
        spec.append((name, qd, pt))
    import torch

    def timed(sp):
        t = ctx.table_from_pages(sp)  # warm: staging, device blocks
        t.close()
        times = []
        for _ in range(args.ingest_reps):
            t0 = time.perf_counter()
            t = ctx.table_from_pages(sp)
            times.append(time.perf_counter() - t0)
            t.close()
        return float(np.median(times))

    # the page buffers as a reader fetches them: into pinned host memory
    # (copied by DMA straight from them), and in pageable memory (staged
    # through the library's pinned buffers by host threads)
    pinned = [(nm, qd, PageTable(torch.from_numpy(np.ascontiguousarray(pt.buf).view(np.uint8)).pin_memory().numpy(),
                                 pt.offsets, pt.lengths, pt.row_counts, pt.null_counts))
              for nm, qd, pt in spec]
    med = timed(pinned)
    med_pageable = timed(spec)
    return {"workload": f"events {n} rows as {rows_per_page}-row pages, 4 columns ({len(starts)} pages each)",
            "page_bytes": int(page_bytes), "ms": med * 1e3, "GB_per_s": page_bytes / med / 1e9,
            "rows_per_s": n / med, "buffers": "pinned host memory",
            "pageable_ms": med_pageable * 1e3, "pageable_GB_per_s": page_bytes / med_pageable / 1e9,
            "reps": args.ingest_reps, "clock": "host, around the synchronous call"}


def run_reference(args, world, rank):
    """Reference arm: the reference's algorithm (oracle port) on the host cores."""
    if rank != 0:
        return
    import oracle
    from querymode_b200 import datagen
    sample = min(args.rows, 20_000_000)
    cols = datagen.events(sample, seed=1)
    q = datagen.events_query()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.run(cols, q, batch_rows=1 << 20, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run(cols, q, batch_rows=1 << 20, threads=threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps * sample * BYTES_PER_ROW / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "i64/f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows_per_step": sample, "bytes_per_row": BYTES_PER_ROW},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{sample:,} rows of {WORKLOAD} per step; the reference's TypeScript/WASM "
                                   "engine cannot run on this image (no node, no zig), its C restatement runs"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import torch

    from querymode_b200 import datagen
    from querymode_b200.engine import Context
    from querymode_b200.query import CQuery

    torch.cuda.set_device(local)
    n = args.rows
    cols = datagen.events(n, seed=1 + rank)
    q = datagen.events_query()
    ctx = Context(local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    table = ctx.table(cols)
    cq = CQuery(q)  # lowered once, like a prepared statement
    bytes_per_query = n * BYTES_PER_ROW

    if world > 1:
        # one query over the union of the ranks' shards: every rank scans its
        # resident shard, the partial group states are gathered to rank 0
        # over NCCL and rank 0 merges them and finalizes
        from querymode_b200.distributed import aggregate_sharded

        def step():
            agg = ctx.aggregate(q)
            try:
                return aggregate_sharded(agg, table, row_offset=rank * n, rows_total=world * n)
            finally:
                agg.close()
    else:
        def step():
            return table.run(cq)

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            res = step()
        barrier(world)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        scan_ms = []
        launches = 0
        with ClockSampler(local) as clocks:
            ev0.record(stream)
            for _ in range(args.steps):
                res = step()
                if res is not None:
                    scan_ms.append(res.stats.scan_ms)
                    launches += res.stats.launches
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier(world)
    elapsed = ev0.elapsed_time(ev1)
    elapsed_max = max_over_ranks(elapsed, world)
    total_bytes = sum_over_ranks(bytes_per_query * args.steps, world)
    value = total_bytes / (elapsed_max / 1e3) / 1e9

    parity = None
    if world == 1 and not args.no_parity:
        parity = check_parity(res, cols, q)

    # roofline of the fused scan kernel (CUDA events around each launch)
    peak, peak_kind = load_peaks()
    scan_avg = float(np.mean(scan_ms)) if scan_ms else float("nan")
    achieved = bytes_per_query / (scan_avg / 1e3) / 1e9
    traffic = profiled_traffic(n)

    # end to end through the C ABI with host inputs in pinned memory
    e2e = None
    if not args.no_e2e:
        pinned = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in cols.items()}
        h2d = sum(v.nbytes for v in pinned.values())
        with torch.cuda.stream(stream):
            t = ctx.table(pinned)
            r = t.run(q)
            t.close()
            d2h = sum(c.values.nbytes for c in r.columns)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.e2e_steps):
                t = ctx.table(pinned)
                r = t.run(q)
                t.close()
            e1.record(stream)
            torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        e2e_val = sum_over_ranks(bytes_per_query * args.e2e_steps, world) / (e2e_ms / 1e3) / 1e9
        e2e = {"value": e2e_val, "unit": "GB/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e2e_ms / args.e2e_steps, "steps": args.e2e_steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(cols, q, min(args.cpu_sample_rows, n))

    configs = None
    if world == 1 and not args.no_configs:
        table.close()
        table = None
        configs = run_configs(ctx, stream, args)

    ingest = None
    if world == 1 and not args.no_ingest:
        ingest = run_ingest(ctx, cols, args)

    batched = None
    if world == 1 and not args.no_batched:
        if table is not None:
            table.close()
            table = None
        batched = run_batched(ctx, stream, local, args)
    serving = None
    if world == 1 and not args.no_serving:
        serving = run_serving(local, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i64/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows_per_gpu": n, "bytes_per_row": BYTES_PER_ROW,
                       "groups": int(res.n_rows), "rows_selected": int(res.stats.rows_selected),
                       "l2": f"inputs {n * BYTES_PER_ROW / 1e9:.2f} GB per GPU > 126 MB L2 (no flush needed)",
                       "parallelism": f"dp{world}" + (" (row shards, partial states gathered to rank 0 over NCCL, merged there)" if world > 1 else "")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "qm_scan_kernel", "kernel_ms": scan_avg},
            "parity": None if parity is None else parity["ok"],
            "parity_check": parity,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "configs": configs,
            "batched": batched,
            "serving": serving,
            "ingest": ingest,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "rows_per_s": n * world * args.steps / (elapsed_max / 1e3),
        }
        print(json.dumps(line), flush=True)
    if table is not None:
        table.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
