"""ws_agg_run_many: several aggregations in one kernel launch (each query its own batches, constants
and result rows; the SMs' CTAs shared out by tiles) give exactly the results of running each query
alone and of the oracle: one compiled plan with different constants over tables of uneven size, and
interpreted queries of different expressions, for the hash, dense private-row and no-key scans."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .helpers import compare_exact

pytestmark = pytest.mark.gpu


def tables():
    rng = np.random.default_rng(21)
    out = []
    for n in (3_000, 250_000, 1_700_000, 700_001):  # uneven sizes, ragged batches
        t = W.Table(n, seg_rows=1 << 18)
        t.add("k", abi.T_I32, rng.integers(0, 40, n, dtype=np.int32))
        t.add("v", abi.T_I64, rng.integers(-10**6, 10**6, n, dtype=np.int64))
        t.add("f", abi.T_F64, rng.random(n))
        t.add("g", abi.T_I32, rng.integers(0, 6, n, dtype=np.int32))  # few groups: the private-row scan
        t.to_device()
        out.append(t)
    return out


def query(t, kind, c, variant=0):
    e = W.env_for(t)
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(1), "BIGINT", True)]
    if kind != "dense":  # (a DOUBLE aggregate over few groups takes the engine's hash path)
        aggs.append(q.Agg("SUM", q.col(2), "DOUBLE", True))
    if variant:
        aggs.append(q.Agg("MAX", q.col(1) * q.ilit(3) + q.ilit(variant), "BIGINT", False))
    keys = [] if kind == "nokeys" else [(q.col(3), True)] if kind == "dense" else [(q.col(0), True)]
    aq = q.AggQuery(e, q.col(1).lt(c), keys, aggs)
    ds = q.dense_spec(aq.plan, [(0, 5)], t.n) if kind == "dense" else None
    assert (ds is not None) == (kind == "dense")
    return e, aq, ds


def fn_of(kind):
    return {"nokeys": abi.JF_NOKEYS, "dense": abi.JF_DENSE, "hash": abi.JF_GROUPED}[kind]


def make(t, e, aq, ds):
    agg = ops.GpuAggregator(aq.plan, 1024, ds)
    agg.add_batches(e.ncols, t.batches(True))
    return agg


@pytest.mark.parametrize("kind", ["hash", "dense", "nokeys"])
@pytest.mark.parametrize("compiled", [True, False], ids=["compiled", "interpreted"])
def test_run_many_equals_alone_and_oracle(kind, compiled):
    ts = tables()
    try:
        qs = [query(t, kind, c, 0 if compiled else i) for i, (t, c) in enumerate(zip(ts, (0, 500_000, -200_000, 10**7)))]
        ops.jit_set_mode(abi.JIT_SYNC if compiled else abi.JIT_OFF)
        jit = ops.jit_get(qs[0][0].env, qs[0][0].ncols, qs[0][1].plan, fn_of(kind), "multi") if compiled else None
        if compiled:
            assert jit
        aggs = [make(t, *qq) for t, qq in zip(ts, qs)]
        ops.agg_run_many(aggs, [qq[0].env for qq in qs], jit)
        for t, (e, aq, ds), agg in zip(ts, qs, aggs):
            assert not agg.overflowed()
            k, a, ex = agg.fetch()
            agg.close()
            alone = make(t, e, aq, ds)
            alone.run(e.env, jit)
            k2, a2, ex2 = alone.fetch()
            alone.close()
            # DOUBLE sums within 1e-12 relative: the launches split the rows over different CTA counts
            compare_exact(aq.plan, k, ex, np.ascontiguousarray(k2).view(np.int64), ex2)
            ok, ow, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols)
            compare_exact(aq.plan, k, ex, ok, ow)
    finally:
        ops.jit_set_mode(-1)
        for t in ts:
            t.free_device()


def test_run_many_rejects_mixed_kinds_and_skips_empty():
    ts = tables()
    try:
        ops.jit_set_mode(abi.JIT_OFF)
        e1, aq1, _ = query(ts[1], "hash", 0)
        e2, aq2, _ = query(ts[2], "nokeys", 0)
        a1, a2 = make(ts[1], e1, aq1, None), make(ts[2], e2, aq2, None)
        with pytest.raises(ops.WsError) as ei:
            ops.agg_run_many([a1, a2], [e1.env, e2.env], None)
        assert ei.value.code == 1210
        a1.close()
        a2.close()
        empty = ops.GpuAggregator(aq1.plan, 1024)  # no batches: skipped
        a1 = make(ts[1], e1, aq1, None)
        ops.agg_run_many([empty, a1], [e1.env, e1.env], None)
        ok, ow, _ = oracle.aggregate(e1.env, aq1.plan, ts[1].batches(False), e1.ncols)
        k, _, ex = a1.fetch()
        compare_exact(aq1.plan, k, ex, ok, ow)
        a1.close()
        empty.close()
    finally:
        ops.jit_set_mode(-1)
        for t in ts:
            t.free_device()
