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
    p.add_argument("--batch-queries", type=int, default=256)
    p.add_argument("--batch-reps", type=int, default=3)
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
    """256 filter -> GROUP BY queries of uneven sizes: one persistent fused
    launch (autotuned, graph-replayed) against the same queries as sequential
    per-query launches."""
    import torch

    from querymode_b200 import autotune, datagen
    from querymode_b200.query import CQuery
    specs = datagen.batch_specs(args.batch_queries, seed=3)
    dev_tables = batch_tables_on_device(specs, local)
    tables = [ctx.table(t) for t in dev_tables]
    cqs = [CQuery(datagen.batch_query(s)) for s in specs]
    batch = ctx.batch(tables, cqs)
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

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            res = table.run(cq)
        barrier(world)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        scan_ms = []
        launches = 0
        with ClockSampler(local) as clocks:
            ev0.record(stream)
            for _ in range(args.steps):
                res = table.run(cq)
                scan_ms.append(res.stats.scan_ms)
                launches += res.stats.launches
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier(world)
    elapsed = ev0.elapsed_time(ev1)
    elapsed_max = max_over_ranks(elapsed, world)
    total_bytes = sum_over_ranks(bytes_per_query * args.steps, world)
    value = total_bytes / (elapsed_max / 1e3) / 1e9

    # roofline of the fused scan kernel (CUDA events around each launch)
    peak, peak_kind = load_peaks()
    scan_avg = float(np.mean(scan_ms))
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

    batched = None
    if world == 1 and not args.no_batched:
        table.close()
        table = None
        batched = run_batched(ctx, stream, local, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i64/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows_per_gpu": n, "bytes_per_row": BYTES_PER_ROW,
                       "groups": int(res.n_rows), "rows_selected": int(res.stats.rows_selected),
                       "l2": f"inputs {n * BYTES_PER_ROW / 1e9:.2f} GB per GPU > 126 MB L2 (no flush needed)",
                       "parallelism": f"dp{world} (independent shards)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "qm_scan_kernel", "kernel_ms": scan_avg},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "batched": batched,
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
