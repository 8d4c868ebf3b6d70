"""The workload pipelines of warpstore_b200.workloads run with the reference's own GPU operators
(oracle/_ref, test infrastructure): the same steps, the same device inputs, so that the tests can
compare results and times stage by stage."""
from __future__ import annotations

import contextlib

from oracle import ref
from warpstore_b200 import abi, ops
from warpstore_b200 import workloads as W


def join_aggregate_run(build: W.Table, probe: W.Table, plans, timer=None):
    """W.join_aggregate_run with the reference's select, gathers, hash join and aggregation."""
    eb, where, ej, aq, ds = plans
    timer = timer or (lambda name: contextlib.nullcontext())
    build.to_device()
    probe.to_device()
    keyv = W.contiguous_view(build, 0, True)
    fkv = W.contiguous_view(probe, 0, True)
    with timer("select"):
        idx, mb, _ = ref.select_multi_dev(eb.env, where, build.batches(True), eb.ncols)
    bkeys = ops.DeviceBuffer(max(mb, 1) * 8)
    with timer("gather build keys"):
        ref.gather(keyv.p, abi.PT_I64, idx, mb, bkeys.ptr)
    with timer("join"):
        ob, op, m, _ = ref.hash_join_dev(abi.ColView(bkeys.ptr, abi.T_I64, 0, 0, 0), mb, fkv, probe.n)
    gk, ct = ops.DeviceBuffer(max(m, 1) * 4), ops.DeviceBuffer(max(m, 1) * 8)
    with timer("gather probe columns"):
        ref.gather(probe.cols[2].dev.ptr, abi.PT_I32, op, m, gk.ptr)
        ref.gather(probe.cols[1].dev.ptr, abi.PT_I64, op, m, ct.ptr)
    with timer("aggregate"):
        keys, accs, _, ovf, _ = ref.aggregate(ej.env, ej.ncols, aq.plan,
                                              [(m, 0, [abi.ColView(gk.ptr, abi.T_I32, 0, 0, 0),
                                                       abi.ColView(ct.ptr, abi.T_I64, 0, 0, 0)])], ds, 1024)
    for p in (idx, ob, op):
        ref.free(p)
    return keys, accs, m


def hash_aggregate_run(batches: list, e, aq, cap: int):
    """W.hash_aggregate_run with the reference's GpuAggregator (same overflow retry)."""
    runs = 0
    while True:
        runs += 1
        keys, accs, g, ovf, _ = ref.aggregate(e.env, e.ncols, aq.plan, batches, None, cap)
        if ovf:
            cap = W.grow_capacity(cap, g)
            continue
        return keys, accs, cap, runs


def distinct_aggregate_run(batches: list, e, aq, dprog, rows_in: int, timer=None):
    """W.distinct_aggregate_run (plain sizing) with the reference's aggregations."""
    timer = timer or (lambda name: contextlib.nullcontext())
    p1 = W.distinct_plans(e, aq, dprog)
    cap1 = 1024
    while cap1 < min(max(rows_in, 1), 1 << 22):
        cap1 <<= 1
    runs = 0
    with timer("phase 1 (keys, x)"):
        while True:
            runs += 1
            kp, ap, g1, ovf, _ = ref.aggregate_compact(e.env, e.ncols, p1, batches, None, cap1)
            if ovf:
                cap1 = W.grow_capacity(cap1, g1)
                continue
            break
    with timer("phase 2 (keys)"):
        env2, nc2, p2 = W.distinct_phase2(aq.plan, p1, kp, ap, g1)
        cap2 = 1024
        while cap2 < 2 * g1:
            cap2 <<= 1
        keys, accs, _, ovf, _ = ref.aggregate(env2, nc2, p2, [(g1, 0, [env2.cols[c] for c in range(nc2)])], None, cap2)
        if ovf:
            raise RuntimeError("phase 2 overflowed a table of twice the pair count")
    ref.free(kp)
    ref.free(ap)
    return keys, accs, runs, g1
