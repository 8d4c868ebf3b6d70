"""High-cardinality hash GROUP BY (Zipf keys, millions of groups) and COUNT(DISTINCT) as the engine
composes it (phase 1 GROUP BY (keys, x), compaction on the device, phase 2 GROUP BY keys): this
library's operators against the CPU oracle (row-exact groups) and against the same pipeline on the
reference's own operators; at full size against an exact numpy restatement of the query and the
reference; the full-size case prints both pipelines' times."""
import time
from contextlib import contextmanager

import numpy as np
import pytest
import torch

from oracle import oracle, ref
from warpstore_b200 import abi, ops
from warpstore_b200 import workloads as W

from . import ref_pipelines as RP

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


def exact_groups_np(t, cut, distinct=False):
    """The full-size query restated in numpy (the oracle's groupby_count_sum_np): sorted by key."""
    key, payload, s = (t.cols[c].data for c in range(3))
    return oracle.groupby_count_sum_np(key, payload, cut, s if distinct else None)


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
        keys, accs, cap, runs = W.hash_aggregate_run(t.batches(True), e, aq, 1 << 14, prog)
    finally:
        ops.jit_set_mode(-1)
    assert runs > 1
    got = engine_arrays(aq, keys, accs)
    ok, ow, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols)
    assert_same(got, oracle_arrays(aq, ok, ow), "ours vs oracle")
    if ref.available():
        rk, ra, _, _ = RP.hash_aggregate_run(t.batches(True), e, aq, cap)
        assert_same(got, engine_arrays(aq, rk, ra), "ours vs reference")


def test_count_distinct_two_phase_matches_oracle_and_reference(small):
    t = small
    e, aq, dprog = W.high_cardinality_query(t, W.high_cardinality_cut(5), distinct=True)
    keys, accs, runs, pairs = W.distinct_aggregate_run(t.batches(True), e, aq, dprog, t.n)
    got = engine_arrays(aq, keys, accs, distinct=True)
    ok, ow, _ = oracle.aggregate_distinct(e.env, aq.plan, dprog, True, t.batches(False), e.ncols)
    assert_same(got, oracle_arrays(aq, ok, ow, distinct=True), "ours vs oracle")
    assert got[3].sum() == pairs
    if ref.available():
        rk, ra, rruns, rpairs = RP.distinct_aggregate_run(t.batches(True), e, aq, dprog, t.n)
        assert rpairs == pairs
        assert_same(got, engine_arrays(aq, rk, ra, distinct=True), "ours vs reference")


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_high_cardinality_full_size_vs_exact_and_reference():
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
        runners = {"ours": lambda: W.hash_aggregate_run(t.batches(True), e, aq, cap, prog),
                   "reference": lambda: RP.hash_aggregate_run(t.batches(True), e, aq, cap)}
        res = {}
        for impl in ("ours", "reference"):
            runners[impl]()  # warm
            with timed((impl, "group by")):
                res[impl] = runners[impl]()
        got = engine_arrays(aq, *res["ours"][:2])
        exact = exact_groups_np(t, cut, distinct=True)
        assert_same(got, exact[:3], "group by: ours vs exact numpy")
        assert_same(got, engine_arrays(aq, *res["reference"][:2]), "group by: ours vs reference")
        ngroups = res["ours"][0].shape[0]

        e2, aq2, dprog = W.high_cardinality_query(t, cut, distinct=True)
        druns = {"ours": lambda timer=None: W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, timer),
                 "reference": lambda timer=None: RP.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, timer)}
        dres = {}
        for impl in ("ours", "reference"):  # warm: plans compiled, the memory pool grown to the largest table
            druns[impl]()
        for impl in ("ours", "reference"):
            @contextmanager
            def stage(name):
                with timed((impl, name)):
                    yield

            dres[impl] = druns[impl](stage)
        # learned sizing of the phase-1 table (ours): same result, fewer overflow reruns
        W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, sizing="learned")  # warm

        @contextmanager
        def lstage(name):
            with timed(("learned", name)):
                yield

        dres["learned"] = W.distinct_aggregate_run(t.batches(True), e2, aq2, dprog, t.n, lstage, sizing="learned")
        assert dres["learned"][3] == dres["ours"][3]
        assert dres["ours"][3] == dres["reference"][3]
        dgot = engine_arrays(aq2, *dres["ours"][:2], distinct=True)
        assert_same(dgot, exact, "count distinct: ours vs exact numpy")
        assert_same(dgot, engine_arrays(aq2, *dres["learned"][:2], distinct=True), "count distinct: learned sizing")
        assert_same(dgot, engine_arrays(aq2, *dres["reference"][:2], distinct=True), "count distinct: ours vs reference")
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
