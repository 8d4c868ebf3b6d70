"""High-cardinality hash GROUP BY (Zipf keys, millions of groups) and COUNT(DISTINCT) as the engine
composes it (phase 1 GROUP BY (keys, x), compaction on the device, phase 2 GROUP BY keys): this
library's operators against the CPU oracle (row-exact groups) and against the same pipeline on the
reference's own operators; the full-size case prints both pipelines' times."""
import time
from contextlib import contextmanager

import numpy as np
import pytest
import torch

from oracle import oracle, ref
from warpstore_b200 import abi, ops
from warpstore_b200 import workloads as W

pytestmark = pytest.mark.gpu


def engine_arrays(aq, keys, accs, distinct=False):
    """Groups of an engine-format result sorted by key: (key, count, exact sum[, distinct count])."""
    a_sum = aq.aggs[1]
    bits = np.ascontiguousarray(accs).view(np.int64)
    k = np.ascontiguousarray(keys).view(np.int64)[:, 0]
    cnt = accs[:, 0].astype(np.int64)
    s = (bits[:, a_sum.hi_slot] << 32) + bits[:, a_sum.slot]  # sums below 2^63 here
    cols = [k, cnt, s] + ([accs[:, -1].astype(np.int64)] if distinct else [])
    order = np.argsort(k, kind="stable")
    return [c[order] for c in cols]


def oracle_arrays(aq, okeys, owords, distinct=False):
    a_sum = aq.aggs[1]
    lo, hi = owords[:, a_sum.slot, 0], owords[:, a_sum.slot, 1]
    assert np.array_equal(hi, lo >> 63), "oracle sums beyond int64 (not expected for these inputs)"
    cols = [okeys[:, 0], owords[:, 0, 0], lo] + ([owords[:, aq.plan.naggs, 0]] if distinct else [])
    order = np.argsort(okeys[:, 0], kind="stable")
    return [c[order] for c in cols]


def assert_same(a, b, what):
    assert len(a[0]) == len(b[0]), f"{what}: group count {len(a[0])} vs {len(b[0])}"
    for i, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"{what}: column {i} differs"


@pytest.fixture(scope="module")
def small():
    t = W.high_cardinality(2_000_000, 200_000, 100_000, seed=5)
    t.to_device()
    yield t
    t.free_device()


@pytest.mark.parametrize("jit", [True, False], ids=["compiled", "interpreted"])
def test_zipf_hash_groupby_matches_oracle_and_reference(small, jit):
    t = small
    e, aq, _ = W.high_cardinality_query(t, W.high_cardinality_cut(5))
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "hc") if jit else None
        # deliberately small first capacity: exercises the overflow retry
        keys, accs, cap, runs = W.hash_aggregate_run(t.batches(True), e, aq, 1 << 14, "ours", prog)
    finally:
        ops.jit_set_mode(-1)
    assert runs > 1
    got = engine_arrays(aq, keys, accs)
    ok, ow, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols)
    assert_same(got, oracle_arrays(aq, ok, ow), "ours vs oracle")
    if ref.available():
        rk, ra, _, _ = W.hash_aggregate_run(t.batches(True), e, aq, cap, "reference")
        assert_same(got, engine_arrays(aq, rk, ra), "ours vs reference")


def test_count_distinct_two_phase_matches_oracle_and_reference(small):
    t = small
    e, aq, dprog = W.high_cardinality_query(t, W.high_cardinality_cut(5), distinct=True)
    keys, accs, runs, pairs = W.distinct_aggregate_run(t.batches(True), e, aq, dprog, t.n, "ours")
    got = engine_arrays(aq, keys, accs, distinct=True)
    ok, ow, _ = oracle.aggregate_distinct(e.env, aq.plan, dprog, True, t.batches(False), e.ncols)
    assert_same(got, oracle_arrays(aq, ok, ow, distinct=True), "ours vs oracle")
    assert got[3].sum() == pairs
    if ref.available():
        rk, ra, rruns, rpairs = W.distinct_aggregate_run(t.batches(True), e, aq, dprog, t.n, "reference")
        assert rpairs == pairs
        assert_same(got, engine_arrays(aq, rk, ra, distinct=True), "ours vs reference")


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_high_cardinality_full_size_vs_reference():
    t = W.high_cardinality()
    t.to_device()
    cut = W.high_cardinality_cut()
    times = {}

    @contextmanager
    def timed(key):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        yield
        torch.cuda.synchronize()
        times[key] = 1e3 * (time.perf_counter() - t0)

    try:
        e, aq, _ = W.high_cardinality_query(t, cut)
        cap = W.plain_capacity(aq.plan, t.n)  # sparse int64 keys: the estimate is the row count
        ops.jit_set_mode(abi.JIT_SYNC)
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "hc")
        ops.jit_set_mode(-1)
        res = {}
        for impl in ("ours", "reference"):
            W.hash_aggregate_run(t.batches(True), e, aq, cap, impl, prog if impl == "ours" else None)  # warm
            with timed((impl, "group by")):
                res[impl] = W.hash_aggregate_run(t.batches(True), e, aq, cap, impl, prog if impl == "ours" else None)
        assert_same(engine_arrays(aq, *res["ours"][:2]), engine_arrays(aq, *res["reference"][:2]), "group by")
        ngroups = res["ours"][0].shape[0]

        e2, aq2, dprog = W.high_cardinality_query(t, cut, distinct=True)
        dres = {}
        for impl in ("ours", "reference"):  # warm: plans compiled, the memory pool grown to the largest table
            W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, impl)
        for impl in ("ours", "reference"):
            @contextmanager
            def stage(name):
                with timed((impl, name)):
                    yield

            dres[impl] = W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, impl, stage)
        # learned sizing of the phase-1 table (ours): same result, fewer overflow reruns
        W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, "ours", sizing="learned")  # warm

        @contextmanager
        def lstage(name):
            with timed(("learned", name)):
                yield

        dres["learned"] = W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, "ours", lstage, sizing="learned")
        assert dres["learned"][3] == dres["ours"][3]
        assert dres["ours"][3] == dres["reference"][3]
        assert_same(engine_arrays(aq2, *dres["ours"][:2], distinct=True),
                    engine_arrays(aq2, *dres["reference"][:2], distinct=True), "count distinct")
        print(f"\n[timing] high-cardinality GROUP BY {t.n} rows, {ngroups} groups, capacity {cap}")
        for s in ("group by", "phase 1 (keys, x)", "phase 2 (keys)"):
            r, o = times[("reference", s)], times[("ours", s)]
            print(f"[timing]   {s:20s} reference {r:9.3f} ms   ours {o:9.3f} ms   ratio {r / o:.2f}x")
        print(f"[timing]   distinct pairs {dres['ours'][3]}, phase-1 runs (overflow retries) {dres['ours'][2]}")
        print(f"[timing]   phase 1 with learned sizing: {times[('learned', 'phase 1 (keys, x)')]:9.3f} ms "
              f"({dres['learned'][2]} run(s)), ratio to the reference "
              f"{times[('reference', 'phase 1 (keys, x)')] / times[('learned', 'phase 1 (keys, x)')]:.2f}x")
    finally:
        t.free_device()
