"""Parity of the GPU aggregation operator (ws_agg_*) with the CPU oracle.

Bit-exact for keys, COUNT, integer SUM (int128), MIN and MAX; DOUBLE SUM within 1e-12 relative.
Each case runs through the C ABI with codegen (NVRTC, sm_100a) and with the on-device interpreter.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .helpers import compare_exact, engine_sum

pytestmark = pytest.mark.gpu


def gpu_aggregate(table, env, plan, dense=None, cap=1024, jit=True, deleted=None, windows=1, fn=None):
    table.to_device()
    if fn is None:
        fn = abi.JF_NOKEYS if plan.nkeys == 0 else abi.JF_DENSE if dense is not None else abi.JF_GROUPED
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        prog = ops.jit_get(env.env, env.ncols, plan, fn, "test") if jit else None
        if jit:
            assert prog, "codegen failed"
        agg = ops.GpuAggregator(plan, cap, dense)
        nb = table.nseg
        per = max(1, (nb + windows - 1) // windows)
        for s in range(nb):
            for i, v in enumerate(table.views(s, True)):
                env.env.cols[i] = v
            agg.add_batch(env.env, env.ncols, table.seg_len(s), deleted[s].ptr if deleted else 0)
            if windows > 1 and (s + 1) % per == 0:
                agg.run_window(env.env, prog)
        agg.run(env.env, prog)
        return agg
    finally:
        ops.jit_set_mode(-1)


def oracle_aggregate(table, env, plan, deleted_host=None):
    batches = table.batches(False, [d.ctypes.data for d in deleted_host] if deleted_host else None)
    return oracle.aggregate(env.env, plan, batches, env.ncols)


def check(table, env, aq, dense=None, cap=1024, deleted=None, deleted_host=None, windows=1):
    ok, ow, _ = oracle_aggregate(table, env, aq.plan, deleted_host)
    for jit in (True, False):
        agg = gpu_aggregate(table, env, aq.plan, dense, cap, jit, deleted, windows)
        assert not agg.overflowed()
        keys, accs, exact = agg.fetch()
        compare_exact(aq.plan, keys, exact, ok, ow)
        agg.close()


# ------------------------------------------------------------------ the benchmark workloads (small)
def test_filter_groupby_hash():
    t = W.filter_groupby_1m(1 << 20, seed=0)
    e, aq = W.filter_groupby_1m_query(t)
    check(t, e, aq)


def test_pricing_summary_dense_exact():
    t = W.pricing_summary(2_500_000, seed=2)
    e, aq, ds = W.pricing_summary_query(t)
    assert ds is not None and ds.G == 6
    check(t, e, aq, dense=ds)
    # the engine-format output recombines to the exact sums
    agg = gpu_aggregate(t, e, aq.plan, ds)
    keys, accs, exact = agg.fetch()
    price = [a for a in aq.aggs if a.fn == "SUM"][1]
    for g in range(accs.shape[0]):
        lo, hi = exact[g, price.slot]
        assert engine_sum(aq.plan, accs[g], price.slot, price.hi_slot) == int(np.uint64(lo)) + (int(hi) << 64)


def test_pricing_summary_as_hash_and_nokeys():
    t = W.pricing_summary(1_200_000, seed=3)
    e, aq, ds = W.pricing_summary_query(t)
    check(t, e, aq, dense=None, cap=64)          # hash GROUP BY on the same query
    e2 = W.env_for(t)
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(2) * (q.ilit(100) - q.col(3)), "BIGINT", False),
            q.Agg("MIN", q.col(2), "BIGINT", True), q.Agg("MAX", q.col(1), "BIGINT", True)]
    aq2 = q.AggQuery(e2, q.col(0).le(2467), [], aggs)
    check(t, e2, aq2)                            # no GROUP BY


# ------------------------------------------------------------------ edge cases
@pytest.mark.parametrize("n", [1, 31, 33, 1023, 1025, (1 << 20) + 5])
def test_ragged_sizes(n):
    rng = np.random.default_rng(n)
    t = W.Table(n)
    t.add("k", abi.T_I32, rng.integers(-3, 5, n, dtype=np.int32))
    t.add("v", abi.T_I64, rng.integers(-10**12, 10**12, n, dtype=np.int64))
    e = W.env_for(t)
    aq = q.AggQuery(e, q.col(1).gt(-10**11), [(q.col(0), True)],
                    [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(1), "BIGINT", True)])
    check(t, e, aq)


def test_sums_beyond_int64_are_exact():
    n = 300_000
    rng = np.random.default_rng(7)
    t = W.Table(n, seg_rows=1 << 17)
    t.add("k", abi.T_I32, rng.integers(0, 3, n, dtype=np.int32))
    t.add("v", abi.T_I64, rng.integers(2**61, 2**62, n, dtype=np.int64))
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True)], [q.Agg("SUM", q.col(1) + q.ilit(1), "BIGINT", False)])
    check(t, e, aq)
    e2 = W.env_for(t)
    aq2 = q.AggQuery(e2, None, [], [q.Agg("SUM", q.col(1), "BIGINT", True)])
    check(t, e2, aq2)
    ds = q.dense_spec(aq.plan, [(0, 2)], n)
    e3 = W.env_for(t)
    aq3 = q.AggQuery(e3, None, [(q.col(0), True)], [q.Agg("SUM", q.col(1), "BIGINT", True)])
    check(t, e3, aq3, dense=q.dense_spec(aq3.plan, [(0, 2)], n))
    assert ds is not None


@pytest.mark.parametrize("where_big", ["first", "middle", "last"])
def test_bounded_sums_switch_to_tested_additions(where_big):
    """Integer sums are added without overflow tests while the arguments stay below the launch's bound,
    and a thread that meets a larger argument tests every later addition: a few huge values (sums past
    int64) among small ones, at the start, middle or end of the scan, in no-key, dense and hash plans;
    products whose operands exceed 32 bits take the tested multiplication (overflow flag included)."""
    n = 1_500_000
    rng = np.random.default_rng(17)
    v = rng.integers(-1000, 1000, n, dtype=np.int64)
    pos = {"first": 0, "middle": n // 2, "last": n - 700}[where_big]
    v[pos:pos + 600] = rng.integers(2**61, 2**62, 600, dtype=np.int64) * rng.choice([-1, 1], 600)
    u = rng.integers(-1000, 1000, n, dtype=np.int64)
    w = rng.integers(1, 50, n, dtype=np.int64)
    w[pos + 100:pos + 110] = 3_000_000_000  # beyond int32: those rows take the tested products
    t = W.Table(n, seg_rows=1 << 18)
    t.add("k", abi.T_I32, rng.integers(0, 5, n, dtype=np.int32))
    t.add("v", abi.T_I64, v)
    t.add("u", abi.T_I64, u)
    t.add("w", abi.T_I64, w)
    for keys in ([], [(q.col(0), True)]):
        e = W.env_for(t)
        aq = q.AggQuery(e, None, keys, [q.Agg("SUM", q.col(1), "BIGINT", True),
                                        q.Agg("SUM", q.col(2) * q.col(3) - q.ilit(7), "BIGINT", False),
                                        q.Agg("SUM", q.col(1) + q.col(2) * q.ilit(3), "BIGINT", False),
                                        q.Agg("COUNT")])
        check(t, e, aq)
        if keys:
            check(t, e, aq, dense=q.dense_spec(aq.plan, [(0, 4)], n))


def test_encoded_columns_nulls_and_deletes():
    n = 700_000
    rng = np.random.default_rng(11)
    t = W.Table(n, seg_rows=1 << 18)
    k = rng.integers(100, 140, n, dtype=np.int32)
    v = rng.integers(-5000, 5000, n, dtype=np.int64)
    vn = v.copy()
    vn[rng.random(n) < 0.1] = abi.NULL_I64
    d = rng.random(n)
    d[rng.random(n) < 0.05] = np.nan
    t.add("k", abi.T_I32, k, enc=1)                 # uint8 + base
    t.add("v", abi.T_I64, v, enc=2)                 # uint16 + base
    t.add("vn", abi.T_I64N, vn, enc=3)              # uint32 + base, NULLs
    t.add("d", abi.T_F64, d)
    e = W.env_for(t)
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("SUM", q.col(2), "BIGINT", True, True),
            q.Agg("MIN", q.col(2), "BIGINT", True, True), q.Agg("MAX", q.col(2), "BIGINT", True, True),
            q.Agg("SUM", q.col(3), "DOUBLE", True, True), q.Agg("MIN", q.col(3), "DOUBLE", True, True),
            q.Agg("COUNT", q.col(2), "BIGINT", True, True)]
    aq = q.AggQuery(e, q.or_(q.col(1).lt(2000), q.col(3).gt(0.5)), [(q.col(0), True)], aggs)
    dels_h, dels_d = [], []
    for s in range(t.nseg):
        m = t.seg_len(s)
        bits = np.zeros((m + 31) // 32, dtype=np.uint32)
        gone = rng.choice(m, m // 20, replace=False)
        np.bitwise_or.at(bits, gone // 32, (np.uint32(1) << (gone % 32).astype(np.uint32)))
        dels_h.append(bits)
        dels_d.append(ops.DeviceBuffer.from_array(bits))
    check(t, e, aq, deleted=dels_d, deleted_host=dels_h)
    ds = q.dense_spec(aq.plan, [(100, 139)], n)
    check(t, e, aq, dense=ds, deleted=dels_d, deleted_host=dels_h)


def test_unaligned_views_use_scalar_loads():
    n = 200_003
    rng = np.random.default_rng(5)
    t = W.Table(n, seg_rows=n)
    t.add("k", abi.T_I32, rng.integers(0, 9, n, dtype=np.int32))
    t.add("v", abi.T_I64, rng.integers(0, 10**9, n, dtype=np.int64))
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True)], [q.Agg("SUM", q.col(1), "BIGINT", True)])
    t.to_device()
    # range scan starting at row 3: raw pointers offset by the caller (not 16-byte aligned)
    off = 3
    views = [abi.ColView(t.cols[0].dev.ptr + 4 * off, abi.T_I32, 0, 0, 0),
             abi.ColView(t.cols[1].dev.ptr + 8 * off, abi.T_I64, 0, 0, 0)]
    hviews = [abi.ColView(t.cols[0].host.ctypes.data + 4 * off, abi.T_I32, 0, 0, 0),
              abi.ColView(t.cols[1].host.ctypes.data + 8 * off, abi.T_I64, 0, 0, 0)]
    ok, ow, _ = oracle.aggregate(e.env, aq.plan, [(n - off, 0, hviews)], e.ncols)
    for jit in (True, False):
        ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED) if jit else None
        agg = ops.GpuAggregator(aq.plan, 64)
        for i, v in enumerate(views):
            e.env.cols[i] = v
        agg.add_batch(e.env, e.ncols, n - off)
        agg.run(e.env, prog)
        keys, accs, ex = agg.fetch()
        compare_exact(aq.plan, keys, ex, ok, ow)
        ops.jit_set_mode(-1)


def test_hash_overflow_then_retry_bigger():
    n = 400_000
    rng = np.random.default_rng(3)
    t = W.Table(n, seg_rows=1 << 17)
    t.add("k", abi.T_I64, rng.integers(0, 50_000, n, dtype=np.int64))
    t.add("v", abi.T_I64, rng.integers(0, 100, n, dtype=np.int64))
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True)], [q.Agg("SUM", q.col(1), "BIGINT", True)])
    cap, tries = 1024, 0
    while True:  # the engine's loop (src/engine_select.cpp:1514-1522): detect, resize, rerun
        agg = gpu_aggregate(t, e, aq.plan, cap=cap)
        if not agg.overflowed():
            break
        want = max(agg.capacity() * 4, agg.group_count() * 4)
        agg.close()
        cap = 1 << (want - 1).bit_length()
        tries += 1
        assert tries < 8
    assert tries >= 1 and cap >= 50_000
    ok, ow, _ = oracle_aggregate(t, e, aq.plan)
    keys, accs, ex = agg.fetch()
    compare_exact(aq.plan, keys, ex, ok, ow)


def test_multi_key_and_double_keys():
    n = 500_000
    rng = np.random.default_rng(9)
    t = W.Table(n, seg_rows=1 << 18)
    t.add("a", abi.T_I32, rng.integers(0, 7, n, dtype=np.int32))
    t.add("b", abi.T_I64, rng.integers(-1, 5, n, dtype=np.int64))    # -1: the empty key word
    t.add("f", abi.T_F64, np.round(rng.random(n) * 4) / 2 - 1.0)     # includes -0.0 / 0.0 after rounding
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True), (q.col(1), True), (q.col(2), False)],
                    [q.Agg("COUNT"), q.Agg("MAX", q.col(2), "DOUBLE", True)])
    check(t, e, aq, cap=4096)
    e2 = W.env_for(t)
    aq2 = q.AggQuery(e2, None, [(q.col(1), True)], [q.Agg("COUNT")])   # key -1 == EMPTY word
    check(t, e2, aq2, cap=64)
    e3 = W.env_for(t)
    aq3 = q.AggQuery(e3, None, [(q.col(2) * q.lit(-1.0), False)], [q.Agg("COUNT")])  # -0.0 groups with 0.0
    check(t, e3, aq3, cap=64)


def test_windows_accumulate():
    t = W.pricing_summary(1_500_000, seed=4)
    e, aq, ds = W.pricing_summary_query(t)
    check(t, e, aq, dense=ds, windows=2)
    check(t, e, aq, dense=None, cap=64, windows=2)


def test_compact_leaves_groups_on_device():
    t = W.filter_groupby_1m(300_000, seed=1)
    e, aq = W.filter_groupby_1m_query(t)
    agg = gpu_aggregate(t, e, aq.plan)
    keys, accs, ex = agg.fetch()
    kp, ap, g = agg.compact()
    dk = ops.device_to_array(kp, np.float64, g * aq.plan.nkeys).reshape(aq.plan.nkeys, g).T
    da = ops.device_to_array(ap, np.float64, g * aq.plan.naggs).reshape(aq.plan.naggs, g).T
    ops.tmp_free(kp)
    ops.tmp_free(ap)
    o1, o2 = np.lexsort(keys.view(np.int64).T[::-1]), np.lexsort(dk.view(np.int64).T[::-1])
    assert np.array_equal(keys[o1].view(np.int64), dk[o2].view(np.int64))
    assert np.array_equal(accs[o1].view(np.int64), da[o2].view(np.int64))


def test_expressions_and_functions():
    n = 300_000
    rng = np.random.default_rng(21)
    t = W.Table(n, seg_rows=1 << 17)
    t.add("d", abi.T_I32, rng.integers(0, 20000, n, dtype=np.int32))      # days since 1970
    t.add("x", abi.T_F64, rng.normal(size=n))
    t.add("c", abi.T_DEC, rng.integers(-10**6, 10**6, n, dtype=np.int64), scale=2)
    e = W.env_for(t)
    yr = q.year(q.col(0))
    case = q.select(q.col(1).gt(0.0), q.ilit(1), q.ilit(0))
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.call1("ABS", q.col(1)), "DOUBLE"),
            q.Agg("SUM", q.col(2), "DECIMAL", True), q.Agg("MAX", q.call1("MONTH", q.col(0)), "DOUBLE"),
            q.Agg("SUM", q.call2("ROUND2", q.col(1), q.ilit(2)), "DOUBLE")]
    aq = q.AggQuery(e, q.and_(q.col(1).ne(q.lit(0.25)), q.not_(q.isnull(q.col(2)))), [(yr, True), (case, True)], aggs)
    check(t, e, aq, cap=256)


def test_add_batches_equals_add_batch():
    t = W.pricing_summary(2_200_000, seed=9)
    e, aq, ds = W.pricing_summary_query(t)
    t.to_device()
    one = gpu_aggregate(t, e, aq.plan, ds)
    k1, a1, x1 = one.fetch()
    agg = ops.GpuAggregator(aq.plan, 1024, ds)
    agg.add_batches(e.ncols, t.batches(True))
    agg.run(e.env, None)
    k2, a2, x2 = agg.fetch()
    o1, o2 = np.lexsort(k1.view(np.int64).T[::-1]), np.lexsort(k2.view(np.int64).T[::-1])
    assert np.array_equal(x1[o1], x2[o2]) and np.array_equal(k1[o1].view(np.int64), k2[o2].view(np.int64))
