"""ws_agg_nokeys_noalloc: the no-GROUP-BY aggregation for callers that may not allocate device memory
(code where the allocator is off limits, or whose memory budget belongs to someone else).  It uses the
library's fixed scratch array instead of allocations; its results must equal the allocating path's
(ws_agg_* with nkeys = 0) and the CPU oracle's on the same inputs, call after call, since every call
reuses the array: also with no batches, a filter no row passes, deleted rows, and rows of many slots
(fewer CTAs fit the array's partial-row area).

Collected last (file name) so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .helpers import DOUBLE_RTOL

pytestmark = pytest.mark.gpu


def table_and_query():
    t = W.pricing_summary(1_500_000, seed=8)
    e = W.env_for(t)
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(2) * (q.ilit(100) - q.col(3)), "BIGINT", False),
            q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(2), "BIGINT", True),
            q.Agg("MAX", q.col(4), "BIGINT", True), q.Agg("SUM", q.col(3) * q.lit(0.5), "DOUBLE", False),
            q.Agg("MAX", q.col(2) * q.lit(0.25), "DOUBLE", False)]
    aq = q.AggQuery(e, q.col(0).le(2000), [], aggs)
    return t, e, aq


def allocating(t, e, aq, prog):
    agg = ops.GpuAggregator(aq.plan, 1)
    for s in range(t.nseg):
        for i, v in enumerate(t.views(s, True)):
            e.env.cols[i] = v
        agg.add_batch(e.env, e.ncols, t.seg_len(s))
    agg.run(e.env, prog)
    _, _, ex = agg.fetch()
    agg.close()
    return ex[0]


def same(aq, got, want):
    for a in range(aq.plan.naggs):
        op, is_int = aq.plan.ops[a], aq.plan.aggInt[a]
        if op == abi.AGG_COUNT or is_int:
            assert got[a, 0] == want[a, 0] and got[a, 1] == want[a, 1], f"slot {a}"
        else:
            g, w = got[a, :1].view(np.float64)[0], want[a, :1].view(np.float64)[0]
            assert g == w or abs(g - w) <= DOUBLE_RTOL * abs(w), f"slot {a}: {g} vs {w}"


@pytest.mark.parametrize("jit", [True, False], ids=["compiled", "interpreted"])
def test_noalloc_matches_allocating_path_twice(jit):
    t, e, aq = table_and_query()
    t.to_device()
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_NOKEYS, "noalloc") if jit else None
        want = allocating(t, e, aq, prog)
        batches = t.batches(True)
        first = ops.agg_nokeys_noalloc(e.env, e.ncols, aq.plan, batches, prog)
        second = ops.agg_nokeys_noalloc(e.env, e.ncols, aq.plan, batches, prog)  # the array is reused
        same(aq, first, want)
        same(aq, second, want)
        assert first[0, 0] > 0
        _, ow, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols)
        same(aq, first, ow[0])
    finally:
        ops.jit_set_mode(-1)
        t.free_device()


def test_noalloc_rejects_oversized_descriptor():
    t, e, aq = table_and_query()
    view = t.views(0, False)  # never dereferenced: the size check comes first
    batches = [(1, 0, view)] * 20_000  # 20,000 batches x 7 columns exceed the fixed 1 MiB descriptor area
    with pytest.raises(ops.WsError) as ei:
        ops.agg_nokeys_noalloc(e.env, e.ncols, aq.plan, batches)
    assert ei.value.code == 1206


def edge_case(kind):
    rng = np.random.default_rng(12)
    n = 700_001
    t = W.Table(n, seg_rows=1 << 18)
    t.add("d", abi.T_I32, rng.integers(0, 2557, n, dtype=np.int32))
    t.add("p", abi.T_I64, rng.integers(-10**12, 10**12, n, dtype=np.int64))
    t.add("x", abi.T_I64, rng.integers(0, 11, n, dtype=np.int64))
    t.add("f", abi.T_F64, rng.random(n))
    e = W.env_for(t)
    deleted = None
    if kind == "many_slots":  # 14 exact sums + min / max: a wide row, so the grid is capped by the part area
        aggs = [q.Agg("SUM", q.col(1) * q.ilit(k + 1) + q.col(2), "BIGINT", False) for k in range(14)]
        aggs += [q.Agg("MIN", q.col(1), "BIGINT", True), q.Agg("MAX", q.col(3), "DOUBLE", True)]
    else:
        aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(2), "BIGINT", True),
                q.Agg("MAX", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(3), "DOUBLE", True),
                q.Agg("SUM", q.col(3), "DOUBLE", True)]
    where = q.col(0).lt(0) if kind == "no_row_passes" else q.col(0).le(2000)
    aq = q.AggQuery(e, where, [], aggs)
    if kind == "deleted":
        deleted = [rng.integers(0, 2**32, (t.seg_len(s) + 31) // 32, dtype=np.uint64).astype(np.uint32)
                   for s in range(t.nseg)]
    return t, e, aq, deleted


@pytest.mark.parametrize("kind", ["no_batches", "no_row_passes", "deleted", "many_slots"])
def test_noalloc_edge_cases_match_allocating_path_and_oracle(kind):
    t, e, aq, deleted = edge_case(kind)
    t.to_device()
    dd = [ops.DeviceBuffer.from_array(d) for d in deleted] if deleted else None
    dev = t.batches(True, [d.ptr for d in dd] if dd else None)
    host = t.batches(False, [d.ctypes.data for d in deleted] if deleted else None)
    if kind == "no_batches":
        dev, host = [], []
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_NOKEYS, "noalloc")
        agg = ops.GpuAggregator(aq.plan, 1)
        if dev:
            agg.add_batches(e.ncols, dev)
        agg.run(e.env, prog)
        _, _, ex = agg.fetch()
        agg.close()
        want = ex[0]
        _, ow, _ = oracle.aggregate(e.env, aq.plan, host, e.ncols)
        for _ in range(2):  # twice: the second call starts from the first one's leftovers
            got = ops.agg_nokeys_noalloc(e.env, e.ncols, aq.plan, dev, prog)
            same(aq, got, want)
            same(aq, got, ow[0])
    finally:
        ops.jit_set_mode(-1)
        t.free_device()
