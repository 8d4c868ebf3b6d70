"""A request loop over resident tables: Poisson arrivals of random filter + GROUP BY queries, admitted
into execution slots as slots and HBM free up, each slot a host thread with its own CUDA stream so the
admitted queries' kernels overlap on the device (continuous batching); latency per query (finish -
arrival), p50 / p99 and QPS.

Two forms with the same results (the tests check every query in the mix against its result alone):
  plain    at most 4 queries in flight, tables sized by the engine's rule (src/engine_select.cpp:1154-1235)
  batched  more slots, admission by the HBM footprint of the queries in flight, hash tables sized by
           the learned estimator (estimator.py; the plain rule stays the overflow fallback)

Tables (config of the serving workload): row counts log-uniform in [min_rows, max_rows]; columns
k1 int32 U[0,8), k2 int32 U[0,1024), k3 int32 U[0,2^20), v int64 U[0,1e6), f float64 U[0,1).
Queries: 1-3 range predicates on v / f / k3 (selectivity 0.1 %-90 %), GROUP BY 1-3 of k1 / k2 / k3
(8 .. 1M groups), COUNT(*), SUM(v), MIN(v), MAX(v), AVG(f).
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import query as q
from .workloads import Table

KEY_CARD = {0: 8, 1: 1024, 2: 1 << 20}  # k1, k2, k3


def make_tables(n_tables: int = 64, min_rows: int = 10_000, max_rows: int = 50_000_000, seed: int = 5) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_tables):
        n = int(np.exp(rng.uniform(np.log(min_rows), np.log(max_rows))))
        t = Table(n)
        t.add("k1", abi.T_I32, rng.integers(0, 8, n, dtype=np.int32))
        t.add("k2", abi.T_I32, rng.integers(0, 1024, n, dtype=np.int32))
        t.add("k3", abi.T_I32, rng.integers(0, 1 << 20, n, dtype=np.int32))
        t.add("v", abi.T_I64, rng.integers(0, 1_000_000, n, dtype=np.int64))
        t.add("f", abi.T_F64, rng.random(n))
        out.append(t)
    return out


@dataclass
class Query:
    qid: int
    table: int
    preds: list            # (column, lo, hi): lo <= col < hi
    keys: list             # GROUP BY key columns (0..2)
    arrival: float = 0.0   # seconds from the start


def make_queries(tables: list, n: int, rate: float, seed: int = 6) -> list:
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        preds = []
        for _ in range(int(rng.integers(1, 4))):
            col = int(rng.choice([2, 3, 4]))  # k3, v, f
            sel = float(np.exp(rng.uniform(np.log(0.001), np.log(0.9))))
            top = {2: 1 << 20, 3: 1_000_000, 4: 1.0}[col]
            lo = rng.uniform(0, top * (1 - sel))
            preds.append((col, lo, lo + top * sel))
        keys = sorted(rng.choice(3, size=int(rng.integers(1, 4)), replace=False).tolist())
        out.append(Query(i, int(rng.integers(0, len(tables))), preds, keys, t))
    return out


def plan_of(t: Table, qr: Query):
    from .workloads import env_for
    e = env_for(t)
    where = None
    for col, lo, hi in qr.preds:
        c = q.col(col)
        lit = (lambda x: q.lit(float(x))) if col == 4 else (lambda x: q.ilit(int(x)))
        p = q.and_(c.ge(lit(lo)), c.lt(lit(hi)))
        where = p if where is None else q.and_(where, p)
    aq = q.AggQuery(e, where, [(q.col(k), True) for k in qr.keys],
                    [q.Agg("COUNT"), q.Agg("SUM", q.col(3), "BIGINT", True), q.Agg("MIN", q.col(3), "BIGINT", True),
                     q.Agg("MAX", q.col(3), "BIGINT", True), q.Agg("SUM", q.col(4), "DOUBLE", False)])
    return e, aq


def plain_capacity_of(qr: Query, rows: int, plan) -> int:
    from .workloads import plain_capacity
    bound = 1
    for k in qr.keys:
        bound *= KEY_CARD[k]
    return plain_capacity(plan, min(bound, rows))


@dataclass
class Result:
    qid: int
    keys: np.ndarray
    exact: np.ndarray
    arrival: float
    start: float = 0.0
    finish: float = 0.0
    runs: int = 1
    cap: int = 0
    checksum: int = 0      # digest of the delivered groups (ws_serve with checksum)
    fsum: float = 0.0
    groups: int = 0


@dataclass
class Prepared:
    """A query compiled ahead of serving (the engine compiles SQL to bytecode before the operators
    run): its expression environment, plan, compiled kernels and plain capacity."""
    qr: Query
    env: object
    ncols: int
    plan: object
    prog: int
    cap: int
    bound: int


def prepare(tables: list, queries: list) -> tuple:
    """(prepared queries, per-table batch arrays); compiles every plan shape the queries use
    (constants live in the environment, so queries differing only in constants share kernels)."""
    from . import estimator, ops
    arrays = [estimator.batch_arrays(t.batches(True)) for t in tables]
    out = []
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        for qr in queries:
            t = tables[qr.table]
            e, aq = plan_of(t, qr)
            prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "serve")
            bound = 1
            for k in qr.keys:
                bound *= KEY_CARD[k]
            out.append(Prepared(qr, e.env, e.ncols, aq.plan, prog, plain_capacity_of(qr, t.n, aq.plan), bound))
    finally:
        ops.jit_set_mode(-1)
    return out, arrays


def execute(p: Prepared, arrays: tuple, learned: bool) -> tuple:
    """One query on the calling thread's stream: (keys, exact words, runs, capacity).  learned: size a
    large table from the estimator (sketch + MLP on the GPU, part of the query's time)."""
    from . import ops
    from .workloads import grow_capacity
    cap = p.cap
    if learned and cap > 1 << 16:  # small tables: the plain rule is already tight
        from . import estimator
        pred = estimator.estimate_groups(p.env, p.ncols, p.plan, arrays, key_range=p.bound)
        cap = min(cap, estimator.learned_capacity(pred))
    nb, bn, bdel, arr, _ = arrays
    runs = 0
    while True:
        runs += 1
        agg = ops.GpuAggregator(p.plan, cap)
        ops.check(ops.lib().ws_agg_add_batches(agg.h, p.ncols, nb, bn, bdel, arr))
        agg.run(p.env, p.prog)
        if agg.overflowed():
            g = agg.group_count()
            agg.close()
            cap = grow_capacity(cap, g)
            continue
        keys, _, ex = agg.fetch()
        agg.close()
        return keys, ex, runs, cap


def footprint(t: Table, qr: Query) -> int:
    """HBM a query holds while it runs (the admission test): its hash table at the plain capacity (rows
    of 8 words) plus batch descriptors and staging."""
    from .workloads import plain_capacity
    shape = abi.AggPlan()
    shape.nkeys, shape.naggs = len(qr.keys), 6
    bound = 1
    for k in qr.keys:
        bound *= KEY_CARD[k]
    return plain_capacity(shape, min(bound, t.n)) * 64 + (1 << 20)


@dataclass
class Stats:
    mode: str
    qps: float
    p50_ms: float
    p99_ms: float
    completed: int
    overflow_reruns: int
    results: dict = field(default_factory=dict)


def run(tables: list, prepared: list, arrays: list, mode: str = "batched", slots: int | None = None,
        hbm_budget: int = 8 << 30, keep_results: bool = True) -> Stats:
    """Serves the prepared queries (arrival times in seconds from the start); tables must be resident."""
    import torch

    from . import ops
    learned = mode == "batched"
    nslots = slots or (16 if learned else 4)
    pending: queue.Queue = queue.Queue()
    done: list = []
    lock = threading.Lock()
    cond = threading.Condition(lock)
    in_flight = [0]
    t0 = time.perf_counter()

    def worker():
        stream = torch.cuda.Stream()
        ops.lib().ws_set_stream(stream.cuda_stream)
        ops.jit_set_mode(abi.JIT_SYNC)
        while True:
            p = pending.get()
            if p is None:
                return
            qr = p.qr
            t = tables[qr.table]
            need = footprint(t, qr)
            with cond:  # admission: the HBM held by the queries in flight stays within the budget
                while in_flight[0] and in_flight[0] + need > hbm_budget:
                    cond.wait()
                in_flight[0] += need
            start = time.perf_counter() - t0
            try:
                keys, ex, runs, cap = execute(p, arrays[qr.table], learned)
            finally:
                with cond:
                    in_flight[0] -= need
                    cond.notify_all()
            r = Result(qr.qid, keys if keep_results else None, ex if keep_results else None, qr.arrival, start,
                       time.perf_counter() - t0, runs, cap)
            with lock:
                done.append(r)

    threads = [threading.Thread(target=worker, daemon=True) for _ in range(nslots)]
    for th in threads:
        th.start()
    for p in prepared:  # arrivals
        delay = p.qr.arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        pending.put(p)
    for _ in threads:
        pending.put(None)
    for th in threads:
        th.join()
    lat = np.array([(r.finish - r.arrival) * 1e3 for r in done])
    span = max(r.finish for r in done) - min(r.arrival for r in done)
    return Stats(mode, len(done) / span, float(np.percentile(lat, 50)), float(np.percentile(lat, 99)), len(done),
                 sum(r.runs - 1 for r in done), {r.qid: r for r in done})


def digest(plan, keys: np.ndarray, exact: np.ndarray) -> tuple:
    """(checksum, DOUBLE SUM total) of a query's groups, ws_serve's digest: the sum (mod 2^64) over the
    groups of mix64 chained over the key bits and the exact words, DOUBLE SUM slots added up apart."""
    from .estimator import mix64
    g = exact.shape[0]
    h = np.full(g, 0x9E3779B97F4A7C15, np.uint64)
    kb = np.ascontiguousarray(keys).view(np.uint64).reshape(g, plan.nkeys) if plan.nkeys else None
    for k in range(plan.nkeys):
        h = mix64(h ^ kb[:, k])
    fs = 0.0
    ex = np.ascontiguousarray(exact).view(np.uint64)
    for a in range(plan.naggs):
        if plan.ops[a] == abi.AGG_SUM and not plan.aggInt[a]:
            fs += float(ex[:, a, 0].view(np.float64).sum())
            continue
        h = mix64(h ^ ex[:, a, 0])
        h = mix64(h ^ ex[:, a, 1])
    return int(h.sum(dtype=np.uint64)), fs


def run_alone(p: Prepared, arrays: list, learned: bool):
    """The query by itself on this thread (the reference result of the mix checks)."""
    keys, ex, _, _ = execute(p, arrays[p.qr.table], learned)
    return keys, ex


def run_native(tables: list, prepared: list, arrays: list, mode: str = "batched", slots: int | None = None,
               hbm_budget: int = 8 << 30, keep_results: bool = True, result_rows: dict | None = None,
               pinned: bool | None = None, arena_bytes: int = 0, checksum: bool = False, batch: int = 0) -> Stats:
    """The same serving loop in the library (ws_serve): C++ worker threads with a CUDA stream each,
    no Python on the per-query path; the prepared queries' arrival times are honoured.

    keep_results: results go to host arrays allocated (and touched) before the loop, result_rows[qid]
    rows each when given, else the key ranges' bound.  Otherwise, with arena_bytes, every worker
    receives its queries' groups in a buffer of its own (reused query after query, as a server's send
    buffer; checksum: each query's groups are digested as they arrive), else they stay on the device.
    batch > 1: arrived queries of one plan share a scan launch, up to `batch` at a time.
    pinned (default: the batched form) selects the one-sync form: result arrays / arenas are pinned
    host memory and the GPU writes the groups into them; plain: pageable memory and the engine's fetch
    sequence."""
    import ctypes as C

    from . import estimator, ops
    learned = mode == "batched"
    pinned = learned if pinned is None else pinned
    nslots = slots or (16 if learned else 4)
    qs = (abi.ServeQuery * len(prepared))()
    keep = []
    for i, p in enumerate(prepared):
        t = tables[p.qr.table]
        nb, bn, bdel, arr, _ = arrays[p.qr.table]
        q = qs[i]
        q.env, q.ncols, q.plan, q.jit = C.addressof(p.env), p.ncols, C.addressof(p.plan), p.prog
        q.nb, q.bn, q.bdel, q.bcols = nb, C.addressof(bn), C.addressof(bdel), C.addressof(arr)
        q.cap_plain, q.key_range, q.arrival_s, q.footprint = p.cap, float(p.bound), p.qr.arrival, footprint(t, p.qr)
        if keep_results:
            g = result_rows[p.qr.qid] if result_rows else min(p.bound, t.n)
            nk, na = p.plan.nkeys, p.plan.naggs
            if pinned:
                hk, hx = ops.HostBuffer((max(g, 1), nk), np.float64), ops.HostBuffer((max(g, 1), na, 2), np.int64)
                keep.append((hk.array, hx.array, hk, hx))
                k, x = hk.array, hx.array
            else:
                k = np.empty((g, nk), np.float64)
                x = np.empty((g, na, 2), np.int64)
                keep.append((k, x))
            k.fill(0)  # page the arrays in before the timed loop
            x.fill(0)
            q.max_groups, q.keys, q.exact = g, k.ctypes.data, x.ctypes.data
        else:
            keep.append(None)
    w = None
    if learned:
        m = estimator.model()
        hold = [np.ascontiguousarray(a) for a in (m.w1, m.b1, m.w2, m.b2, m.w3, m.mean, m.std)]
        keep.append(hold)
        w = abi.EstimatorWeights(estimator.HIDDEN, hold[0].ctypes.data, hold[1].ctypes.data, hold[2].ctypes.data,
                                 hold[3].ctypes.data, hold[4].ctypes.data, float(m.b3), hold[5].ctypes.data,
                                 hold[6].ctypes.data, m.margin(), m.gate)
    wall = C.c_double()
    opt = abi.ServeOptions(nslots, hbm_budget, C.addressof(w) if w else None, int(bool(pinned)),
                           0 if keep_results else int(arena_bytes), int(bool(checksum)), int(batch))
    ops.check(ops.lib().ws_serve(qs, len(prepared), C.byref(opt), C.byref(wall)))
    lat = np.array([(q.finish_s - q.arrival_s) * 1e3 for q in qs])
    span = max(q.finish_s for q in qs) - min(q.arrival_s for q in qs)
    results = {}
    for i, p in enumerate(prepared):
        q = qs[i]
        k, x = keep[i][:2] if keep[i] is not None else (None, None)
        results[p.qr.qid] = Result(p.qr.qid, k[:q.groups].copy() if k is not None else None,
                                   x[:q.groups].copy() if x is not None else None, q.arrival_s, q.start_s, q.finish_s,
                                   q.runs, q.cap_used, int(q.checksum), float(q.fsum), int(q.groups))
    return Stats(mode, len(prepared) / span, float(np.percentile(lat, 50)), float(np.percentile(lat, 99)),
                 len(prepared), sum(q.runs - 1 for q in qs), results)


def main():
    """Serving measurement: both forms over the same tables and arrivals, each query's groups delivered
    to a per-worker buffer and digested, the digests of the two forms compared query by query (DOUBLE
    SUM totals within 1e-9 relative, the rest exact).  One JSON line per form and repeat.

        python -m warpstore_b200.serving [--tables 64] [--max-rows 5e7] [--queries 10000] [--rate 2000]
    """
    import argparse
    import json

    import torch

    from . import ops
    ap = argparse.ArgumentParser()
    ap.add_argument("--tables", type=int, default=64)
    ap.add_argument("--min-rows", type=float, default=1e4)
    ap.add_argument("--max-rows", type=float, default=5e7)
    ap.add_argument("--queries", type=int, default=10_000)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--arena-mb", type=int, default=256, help="per-worker result buffer")
    ap.add_argument("--hbm-gb", type=float, default=8.0, help="admission budget")
    ap.add_argument("--batch", type=int, default=8,
                    help="a third form: batched, with up to this many arrived queries of one plan per launch (<= 1: none)")
    a = ap.parse_args()
    t0 = time.perf_counter()
    tables = make_tables(a.tables, int(a.min_rows), int(a.max_rows), seed=5)
    for t in tables:
        t.to_device()
    queries = make_queries(tables, a.queries, rate=a.rate, seed=6)
    prepared, arrays = prepare(tables, queries)
    rows = sum(t.n for t in tables)
    setup_s = time.perf_counter() - t0
    ops.jit_set_mode(abi.JIT_SYNC)
    kw = dict(keep_results=False, arena_bytes=a.arena_mb << 20, checksum=True, hbm_budget=int(a.hbm_gb * 2 ** 30))
    try:
        run_native(tables, prepared[:200], arrays, "batched", **kw)  # warm: pools, pinned buffers, weights
        run_native(tables, prepared[:200], arrays, "plain", **kw)
        ref = None
        for rep in range(a.repeats):
            for mode, batch in [("plain", 1), ("batched", 1)] + ([("batched", a.batch)] if a.batch > 1 else []):
                torch.cuda.synchronize()
                st = run_native(tables, prepared, arrays, mode, batch=batch, **kw)
                dig = {qid: (r.checksum, r.fsum, r.cap) for qid, r in st.results.items()}
                same = None
                if ref is not None:
                    same = all(dig[q][0] == ref[q][0] and abs(dig[q][1] - ref[q][1]) <= 1e-9 * max(abs(ref[q][1]), 1e-300)
                               for q in ref)
                else:
                    ref = dig
                print(json.dumps({"form": mode, "batch": batch, "repeat": rep, "qps": round(st.qps, 1),
                                  "p50_ms": round(st.p50_ms, 3),
                                  "p99_ms": round(st.p99_ms, 3), "completed": st.completed,
                                  "overflow_reruns": st.overflow_reruns,
                                  "groups": int(sum(r.groups for r in st.results.values())),
                                  "digests_equal_first_run": same,
                                  "config": {"tables": a.tables, "rows": rows, "queries": a.queries,
                                             "rate_per_s": a.rate, "arena_mb": a.arena_mb,
                                             "slots": 16 if mode == "batched" else 4, "setup_s": round(setup_s, 1)}}),
                      flush=True)
    finally:
        ops.jit_set_mode(-1)
        for t in tables:
            t.free_device()


if __name__ == "__main__":
    main()
