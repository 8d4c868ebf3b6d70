#!/usr/bin/env python
"""Benchmark of the B200 query-execution core.

Default workload: the pricing-summary scan (60,000,000 rows in 2^20-row segments; filter + dense
GROUP BY over 2 one-byte dictionary-coded flags; exact int128 sums of price and price expressions),
the configuration the headline metric is quoted on.  One step = one query: build the aggregator,
add the 58 segment batches, one fused scan kernel, compaction and the groups written into pinned host
memory (ws_agg_fetch_async), checked on the host.  Query i is queued before query i - 1 is checked, so
the GPU does not wait for the host between queries.

  value   device-timed throughput (G rows/s) with the table resident in HBM (2.28 GB of inputs, far
          larger than the 126 MB L2, so no flush between steps is needed)
  e2e     the same query through the C ABI from pinned host buffers: every step copies the segment
          columns host -> device and reads the groups back
  roofline  the scan kernel's algorithmic bytes (38 B/row) per launch / its CUDA-event duration
  cpu_baseline  the CPU oracle (C++ restatement, all host threads) on a bounded sample

`--impl reference` times the reference's CPU path: the reference has no CPU implementation of these
operators, so the CPU oracle port stands in (kind "port").
Multi-GPU (torchrun): every rank runs its own replica of the workload (the operators do not shard a
query across GPUs); value = rows of all ranks / max step time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per row of the workload's scan kernel, from one ncu capture of a smaller
# case of the same kernel (8,388,608 and 25,000,000 rows), scaled to a launch by its rows: the traffic
# grows in proportion to the rows scanned
NCU_DRAM_BYTES_PER_ROW = {"pricing_summary_60m": 38.52, "high_cardinality_100m": 22.94, "pricing_nokeys_60m": 28.55}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for i, nm in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def reduce_max(x: float, ws: int, device: str = "cuda") -> float:
    """Max over ranks (the step time of the slowest replica)."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(rows_per_rank: int, ws: int, ms_step_max: float) -> float:
    """G rows/s of all replicas: every rank scans rows_per_rank per step; the job's step lasts as long
    as the slowest rank's."""
    return rows_per_rank * ws / (ms_step_max / 1e3) / 1e9


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------ CPU baseline (oracle)
def cpu_oracle_rate(table, env, plan, budget_s: float, max_segments: int = 8):
    """Rows/s of the oracle over the first segments of the table, repeated for about budget_s."""
    from oracle import oracle
    nseg = min(max_segments, table.nseg)
    batches = table.batches(False)[:nseg]
    rows = sum(b[0] for b in batches)
    done, t0 = 0, time.perf_counter()
    while True:
        oracle.aggregate(env.env, plan, batches, env.ncols)
        done += rows
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return done / el, rows, os.cpu_count() or 1


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def make_checker(name: str, table, env, aq, rank: int):
    """(check(keys, exact, groups) -> None or what differs, description, every_step): the oracle's
    groups of the whole workload, computed once before timing, against which results are compared
    outside the timed events.  Few groups: every timed step; the high-cardinality workload (4M groups,
    seconds to compare): the last timed step."""
    from oracle import oracle
    if name == "high_cardinality_100m":
        from warpstore_b200 import workloads as W
        key, payload = table.cols[0].data, table.cols[1].data
        cut = W.high_cardinality_cut(4 + rank)  # the workload's predicate constant (make_workload)
        wk, wc, ws_ = oracle.groupby_count_sum_np(key, payload, cut)
        a_sum = aq.aggs[1]

        def check(keys, exact, g):
            if g != wk.size:
                return f"{g} groups, the numpy restatement has {wk.size}"
            k = np.ascontiguousarray(keys[:g, 0]).view(np.int64)
            o = np.argsort(k)
            if not np.array_equal(k[o], wk):
                return "group keys differ"
            ex = exact[:g][o]
            if not np.array_equal(ex[:, 0, 0], wc):
                return "COUNT differs"
            lo, hi = ex[:, a_sum.slot, 0], ex[:, a_sum.slot, 1]
            if not (np.array_equal(lo, ws_) and np.array_equal(hi, ws_ >> 63)):
                return "SUM differs (exact words)"
            return None
        return check, "numpy restatement (sort + exact int64 sums), last timed step", False
    okeys, owords, _ = oracle.aggregate(env.env, aq.plan, table.batches(False), env.ncols)
    return (lambda keys, exact, g: oracle.compare_groups(aq.plan, okeys, owords, keys, exact, g),
            "oracle (C++ restatement, int128 words), every timed step", True)


# ------------------------------------------------------------------ workloads
def make_workload(name: str, rank: int, rows: int | None = None):
    from warpstore_b200 import workloads as W
    if name == "pricing_summary_60m":
        t = W.pricing_summary(rows or W.PRICING_ROWS, seed=2 + rank)
        e, aq, ds = W.pricing_summary_query(t)
        return t, e, aq, ds, W.PRICING_BYTES_PER_ROW, 1024, {
            "workload": "pricing_summary_60m", "rows": t.n, "segments": t.nseg, "segment_rows": t.seg_rows,
            "columns": "ship_date i32, quantity/price/discount/tax i64, flag1/flag2 u8-encoded",
            "groups": 6, "aggregation": "dense",
            "l2": f"inputs {t.n * W.PRICING_BYTES_PER_ROW / 1e9:.2f} GB > 126 MB L2 (no flush needed)"}
    if name == "pricing_nokeys_60m":  # the same table, filter + aggregates without GROUP BY
        from warpstore_b200 import query as q
        t = W.pricing_summary(rows or W.PRICING_ROWS, seed=2 + rank)
        e = W.env_for(t)
        aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(2) * (q.ilit(100) - q.col(3)), "BIGINT", False),
                q.Agg("MIN", q.col(2), "BIGINT", True), q.Agg("MAX", q.col(1), "BIGINT", True)]
        aq = q.AggQuery(e, q.col(0).le(2467), [], aggs)
        return t, e, aq, None, 4 + 8 * 3, 1, {
            "workload": "pricing_nokeys_60m", "rows": t.n, "segments": t.nseg, "segment_rows": t.seg_rows,
            "columns": "ship_date i32, price/discount/quantity i64 (28 B/row read)", "groups": 1,
            "aggregation": "no keys: COUNT, exact SUM(price*(100-discount)), MIN(price), MAX(quantity)",
            "l2": f"inputs {t.n * 28 / 1e9:.2f} GB > 126 MB L2 (no flush needed)"}
    if name == "high_cardinality_100m":
        n = rows or W.HC_ROWS
        t = W.high_cardinality(n, W.HC_RANKS if n == W.HC_ROWS else max(n // 10, 1000), W.HC_DICT, seed=4 + rank)
        e, aq, _ = W.high_cardinality_query(t, W.high_cardinality_cut(4 + rank))
        return t, e, aq, None, W.HC_BYTES_PER_ROW, W.plain_capacity(aq.plan, t.n), {
            "workload": "high_cardinality_100m", "rows": t.n, "segments": t.nseg, "segment_rows": t.seg_rows,
            "columns": "key i64 (Zipf s=1.1 over 10M ranks, mixed), payload i64, s i32",
            "aggregation": "hash", "l2": f"inputs {t.n * 20 / 1e9:.2f} GB > 126 MB L2 (no flush needed)"}
    if name == "filter_groupby_1m":
        t = W.filter_groupby_1m(1 << 20, seed=0 + rank)
        e, aq = W.filter_groupby_1m_query(t)
        return t, e, aq, None, W.FILTER_GROUPBY_BYTES_PER_ROW, 1024, {
            "workload": "filter_groupby_1m", "rows": t.n, "groups": 16, "aggregation": "hash",
            "l2": "inputs 21 MB fit in L2: L2 flushed between steps"}
    raise SystemExit(f"unknown workload {name}")


def run_ours(args, ws, rank, local):
    import torch

    from warpstore_b200 import abi, estimator, ops

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    ops.lib().ws_set_stream(stream.cuda_stream)
    ops.gpu_init()
    table, env, aq, ds, bpr, cap, cfg = make_workload(args.workload, rank, args.rows)
    # the exact groups of the whole workload, computed on the host before timing: every result is
    # compared with them outside the timed events (a mismatch ends the run with an error)
    check, verified, check_every = make_checker(args.workload, table, env, aq, rank)
    table.to_device()
    ops.jit_set_cache_dir(os.path.join(tempfile.gettempdir(), "warpstore_b200_plans"))
    ops.jit_set_mode(abi.JIT_SYNC)
    fn = abi.JF_NOKEYS if aq.plan.nkeys == 0 else abi.JF_DENSE if ds is not None else abi.JF_GROUPED
    prog = ops.jit_get(env.env, env.ncols, aq.plan, fn, cfg["workload"])
    if not prog:
        raise SystemExit("codegen failed")
    flush = None
    if table.nbytes() < 512 << 20:  # small inputs: write a buffer larger than L2 between steps
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    batches = table.batches(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    arrays = estimator.batch_arrays(batches)
    max_groups = ds.G if ds is not None else cap
    nk, na = aq.plan.nkeys, aq.plan.naggs
    # two result slots in pinned host memory: query i writes slot i % 2 while query i - 1 is checked
    slots = [(ops.HostBuffer((max_groups, max(nk, 1)), np.float64), ops.HostBuffer((max_groups, na, 2), np.int64),
              ops.HostBuffer(1, ops.FETCH_STATUS), torch.cuda.Event()) for _ in range(2)]

    def queue_step(i=None, slot=0):
        """Queues one query (aggregator, batches, the scan, compaction + groups into pinned memory)."""
        agg = ops.GpuAggregator(aq.plan, cap, ds)
        ops.check(ops.lib().ws_agg_add_batches(agg.h, env.ncols, *arrays[:4]))
        with torch.cuda.stream(stream):
            if i is not None:
                ev[i][0].record(stream)
            agg.run(env.env, prog)
            if i is not None:
                ev[i][1].record(stream)
        hk, hx, st, done = slots[slot]
        agg.fetch_async(max_groups, hk if nk else None, hx, st)
        done.record(stream)
        return agg, slot

    def finish_step(q, verify=check_every):
        """Waits for a queued query and checks its status word and (verify) its groups."""
        agg, slot = q
        hk, hx, st, done = slots[slot]
        done.synchronize()
        s = st.array[0]
        if s["error"] or s["overflow"] or s["groups"] > max_groups or s["groups"] < 1:
            raise SystemExit(f"query failed: status {s}")
        agg.close()
        if verify:
            err = check(hk.array if nk else None, hx.array, int(s["groups"]))
            if err:
                raise SystemExit(f"result differs from the {verified.split(',')[0]}: {err}")
        return int(s["groups"])

    def step(i=None):
        return finish_step(queue_step(i))

    def maybe_flush():
        if flush is not None:
            with torch.cuda.stream(stream):
                flush.fill_(1)

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        maybe_flush()
        step()
    soak = time.perf_counter()
    while time.perf_counter() - soak < args.soak:  # untimed steps so the clock samples see the load
        maybe_flush()
        step()
    stream.synchronize()
    barrier(ws)
    t_total = 0.0
    launches0 = ops.kernel_launches()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    prev = None
    for i in range(args.steps):  # query i is queued before query i - 1 is checked: the GPU never waits
        maybe_flush()             # for the host between queries
        if i == 0:
            s0.record(stream)
        cur = queue_step(i, i % 2)
        if prev is not None:
            finish_step(prev)
        prev = cur
    s1.record(stream)               # after the last query's work, before its host-side check
    finish_step(prev, verify=True)  # the last step is verified in every mode
    s1.synchronize()
    launches = ops.kernel_launches() - launches0
    total_ms = s0.elapsed_time(s1)
    if flush is not None:  # the flush kernels are not query work
        total_ms = sum(a.elapsed_time(b) for a, b in ev) + 0.0
    barrier(ws)
    kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    ms_step = reduce_max(total_ms / args.steps, ws)
    rows_all = table.n * ws
    value = whole_job_rate(table.n, ws, ms_step)

    # end to end from pinned host buffers through the C ABI
    e2e_steps = max(1, min(args.steps, 5))
    hosts = [torch.from_numpy(c.host).pin_memory() for c in table.cols]
    devs = [torch.empty(c.host.size, dtype=torch.uint8, device="cuda") for c in table.cols]
    e2e_batches = []
    for s in range(table.nseg):
        views = table.views(s, True)
        for c, v in enumerate(views):
            v.p = devs[c].data_ptr() + table.cols[c].offsets[s]
        e2e_batches.append((table.seg_len(s), 0, views))
    d2h = 0

    e2e_arrays = estimator.batch_arrays(e2e_batches)

    def e2e_step():
        nonlocal d2h
        with torch.cuda.stream(stream):
            for h, d in zip(hosts, devs):
                d.copy_(h, non_blocking=True)
        agg = ops.GpuAggregator(aq.plan, cap, ds)
        ops.check(ops.lib().ws_agg_add_batches(agg.h, env.ncols, *e2e_arrays[:4]))
        agg.run(env.env, prog)
        hk, hx, st, done = slots[0]
        agg.fetch_async(max_groups, hk if nk else None, hx, st)
        ops.sync()
        g = int(st.array[0]["groups"])
        if st.array[0]["error"] or st.array[0]["overflow"] or not 1 <= g <= max_groups:
            raise SystemExit(f"query failed: status {st.array[0]}")
        d2h = g * 8 * (nk + 2 * na) + ops.FETCH_STATUS.itemsize
        agg.close()
        if check_every:
            err = check(hk.array if nk else None, hx.array, g)
            if err:
                raise SystemExit(f"end-to-end result differs from the {verified.split(',')[0]}: {err}")

    e2e_step()
    stream.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1) / e2e_steps, ws)
    clk = clocks.stop()
    e2e_value = rows_all / (e2e_ms / 1e3) / 1e9

    peak, peak_kind = measured_peak()
    algo_bytes = bpr * table.n
    traffic = args.traffic
    if traffic is None and cfg["workload"] in NCU_DRAM_BYTES_PER_ROW:
        traffic = round(NCU_DRAM_BYTES_PER_ROW[cfg["workload"]] * table.n)
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rate, rows, cores = cpu_oracle_rate(table, env, aq.plan, args.cpu_seconds)
        cpu = {"value": rate / 1e9, "unit": "G rows/s", "cores": cores, "cpu": cpu_model(), "kind": "port",
               "sample": f"{rows} rows (first segments of the same table), repeated for ~{args.cpu_seconds:.0f} s"}
    if rank == 0:
        line = {
            "metric": "scan_filter_aggregate_throughput", "value": round(value, 4), "unit": "G rows/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded numpy)", "config": dict(cfg, parallelism=f"replicas{ws}"),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": f"{peak_kind} hbm_gbs",
                         "kernel_ms": round(kernel_ms, 4), "algorithmic_bytes": algo_bytes},
            "e2e": {"value": round(e2e_value, 4), "unit": "G rows/s", "h2d_bytes_per_step": table.nbytes(),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": cpu, "verified": verified,
        }
        print(json.dumps(line), flush=True)
    table.free_device()


def run_reference(args, ws, rank, local):
    if rank != 0:
        return
    from oracle import oracle
    from warpstore_b200 import query as q
    from warpstore_b200 import workloads as W
    q.TYPER = oracle.prog_is_int  # plans typed by the oracle: this arm loads none of the library's code
    name = args.workload
    if name == "pricing_summary_60m":
        # the per-step sample: 8 segments (8.4M rows) of the same table
        t = W.pricing_summary(8 * W.SEG_ROWS, seed=2)
        e, aq, ds = W.pricing_summary_query(t)
        cfg = {"workload": "pricing_summary_60m", "rows": W.PRICING_ROWS, "sample_rows": t.n}
    else:
        t = W.filter_groupby_1m(1 << 20, seed=0)
        e, aq = W.filter_groupby_1m_query(t)
        cfg = {"workload": "filter_groupby_1m", "rows": t.n, "sample_rows": t.n}
    batches = t.batches(False)
    for _ in range(args.warmup):
        oracle.aggregate(e.env, aq.plan, batches, e.ncols)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.aggregate(e.env, aq.plan, batches, e.ncols)
    el = time.perf_counter() - t0
    rate = t.n * args.steps / el / 1e9
    cores = os.cpu_count() or 1
    line = {"metric": "scan_filter_aggregate_throughput", "value": round(rate, 4), "unit": "G rows/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded numpy)", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": round(rate, 4), "unit": "G rows/s", "cores": cores, "cpu": cpu_model(), "kind": "port",
                             "sample": f"{t.n} rows per step"},
            "e2e": {"value": round(rate, 4), "unit": "G rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pricing_summary_60m",
                    choices=["pricing_summary_60m", "pricing_nokeys_60m", "filter_groupby_1m", "high_cardinality_100m"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic", type=float, default=None, help="ncu dram bytes per launch, when known")
    ap.add_argument("--rows", type=int, default=None, help="pricing workload rows (default 60,000,000)")
    ap.add_argument("--soak", type=float, default=1.0, help="seconds of untimed steps before timing")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, ws, rank, 0)
        return
    ws, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
