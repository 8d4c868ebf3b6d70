"""Prepared queries (ws_exec_*): a query built once with a CUDA graph and run with new constants each
time gives exactly the groups of the ordinary path (create / add / run / fetch) for the same
constants — hash, dense and no-key plans; overflow is reported in the status; other expressions are
refused.  Prints the per-query latency of the three forms on the 1M-row filter + GROUP BY.  A group of
prepared queries of one plan (one graph, one multi-query scan) gives each query's groups as alone."""
import ctypes
import struct
import time

import numpy as np
import pytest

from warpstore_b200 import abi, ops
from warpstore_b200 import estimator as E
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

pytestmark = pytest.mark.gpu


def const_index(env, value: int) -> int:
    want = struct.pack("<q", value)
    for i in range(abi.MAX_CONSTS):
        if struct.pack("<d", env.consts[i]) == want:
            return i
    raise AssertionError(f"constant {value} not in the environment")


def set_int_const(env, i: int, value: int):
    env.consts[i] = struct.unpack("<d", struct.pack("<q", value))[0]


def ordinary(plan, cap, dense, env, ncols, arrays, prog):
    agg = ops.GpuAggregator(plan, cap, dense)
    ops.check(ops.lib().ws_agg_add_batches(agg.h, ncols, *arrays[:4]))
    agg.run(env, prog)
    ovf = agg.overflowed()
    keys, _, ex = agg.fetch() if not ovf else (None, None, None)
    agg.close()
    return ovf, keys, ex


def dsum_slots(plan):
    return [a for a in range(plan.naggs) if plan.ops[a] == abi.AGG_SUM and not plan.aggInt[a]]


def same_groups(plan, k, x, rk, rx):
    assert np.array_equal(k.view(np.int64), rk.view(np.int64))
    d = dsum_slots(plan)
    exact = [a for a in range(plan.naggs) if a not in d]
    assert np.array_equal(x[:, exact], rx[:, exact])
    for a in d:  # DOUBLE SUM: the order of the atomic additions may change the last bits
        np.testing.assert_allclose(x[:, a, 0].view(np.float64), rx[:, a, 0].view(np.float64), rtol=1e-12)


@pytest.fixture(scope="module")
def fg():
    t = W.filter_groupby_1m(1 << 20, seed=0)
    t.to_device()
    yield t
    t.free_device()


def test_runs_with_new_constants_equal_the_ordinary_path(fg):
    e, aq = W.filter_groupby_1m_query(fg)
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "exec")
        arrays = E.batch_arrays(fg.batches(True))
        ex = ops.Executor(aq.plan, 1024, None, e.env, e.ncols, arrays, prog, 64)
        ci = const_index(e.env, 500_000)
        for cut in (500_000, 1, 999_999, 250_000, 0, 500_000):
            set_int_const(e.env, ci, cut)
            ex.run(e.env)
            ops.sync()
            k, x, st = ex.results()
            ovf, rk, rx = ordinary(aq.plan, 1024, None, e.env, e.ncols, arrays, prog)
            assert not ovf and st["overflow"] == 0 and st["error"] == 0
            assert st["groups"] == rk.shape[0]
            same_groups(aq.plan, k, x, rk, rx)
        # other expressions are refused
        e2, _ = W.filter_groupby_1m_query(fg)
        e2.env.code[0].op = (e2.env.code[0].op + 1) % 250
        with pytest.raises(ops.WsError) as ei:
            ex.run(e2.env)
        assert ei.value.code == 1210
        ex.close()
    finally:
        ops.jit_set_mode(-1)


def test_dense_nokeys_and_overflow():
    t = W.pricing_summary(1_500_000, seed=7)
    t.to_device()
    e, aq, ds = W.pricing_summary_query(t)
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        arrays = E.batch_arrays(t.batches(True))
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_DENSE, "exec")
        ex = ops.Executor(aq.plan, 1024, ds, e.env, e.ncols, arrays, prog, 16)
        ci = const_index(e.env, 2467)
        for day in (2467, 100, 2556):
            set_int_const(e.env, ci, day)
            ex.run(e.env)
            ops.sync()
            k, x, st = ex.results()
            _, rk, rx = ordinary(aq.plan, 1024, ds, e.env, e.ncols, arrays, prog)
            assert st["groups"] == rk.shape[0]
            same_groups(aq.plan, k, x, rk, rx)
        ex.close()
        e2 = W.env_for(t)
        aq2 = q.AggQuery(e2, q.col(0).le(2467), [], [q.Agg("COUNT"), q.Agg("SUM", q.col(2), "BIGINT", True)])
        prog2 = ops.jit_get(e2.env, e2.ncols, aq2.plan, abi.JF_NOKEYS, "exec")
        ex2 = ops.Executor(aq2.plan, 1, None, e2.env, e2.ncols, arrays, prog2, 1)
        ex2.run(e2.env)
        ops.sync()
        k, x, st = ex2.results()
        _, rk, rx = ordinary(aq2.plan, 1, None, e2.env, e2.ncols, arrays, prog2)
        assert st["groups"] == 1 and np.array_equal(x, rx)
        ex2.close()
        # a hash table too small: the status says so
        e3 = W.env_for(t)
        aq3 = q.AggQuery(e3, None, [(q.col(2), True)], [q.Agg("COUNT")])
        prog3 = ops.jit_get(e3.env, e3.ncols, aq3.plan, abi.JF_GROUPED, "exec")
        ex3 = ops.Executor(aq3.plan, 1024, None, e3.env, e3.ncols, arrays, prog3, 4096)
        ex3.run(e3.env)
        ops.sync()
        _, _, st = ex3.results()
        assert st["overflow"] == 1
        ex3.close()
    finally:
        ops.jit_set_mode(-1)
        t.free_device()


def test_latency_of_the_three_forms(fg):
    e, aq = W.filter_groupby_1m_query(fg)
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "exec")
        arrays = E.batch_arrays(fg.batches(True))
        ex = ops.Executor(aq.plan, 1024, None, e.env, e.ncols, arrays, prog, 64)
        hk, hx = ops.HostBuffer((64, 1), np.float64), ops.HostBuffer((64, aq.plan.naggs, 2), np.int64)
        hs = ops.HostBuffer(1, ops.FETCH_STATUS)
        n = 200

        def engine():
            ordinary(aq.plan, 1024, None, e.env, e.ncols, arrays, prog)

        def one_sync():
            agg = ops.GpuAggregator(aq.plan, 1024)
            ops.check(ops.lib().ws_agg_add_batches(agg.h, e.ncols, *arrays[:4]))
            agg.run(e.env, prog)
            agg.fetch_async(64, hk, hx, hs)
            ops.sync()
            agg.close()

        def graph():
            ex.run(e.env)
            ops.sync()

        out = {}
        for name, fn in (("engine sequence", engine), ("one-sync", one_sync), ("prepared graph", graph)):
            for _ in range(20):
                fn()
            t0 = time.perf_counter()
            for _ in range(n):
                fn()
            out[name] = (time.perf_counter() - t0) / n * 1e6
        print("\n[exec] 1M-row filter + GROUP BY, per query: " +
              ", ".join(f"{k} {v:.0f} us" for k, v in out.items()))
        assert out["prepared graph"] < out["engine sequence"]
        ex.close()
        for b in (hk, hx, hs):
            b.close()
    finally:
        ops.jit_set_mode(-1)


@pytest.mark.parametrize("kind", ["hash", "dense", "nokeys"])
def test_group_of_prepared_queries_equals_each_alone(kind):
    """Prepared queries of one compiled plan over tables of uneven size, run as one group (one graph,
    one multi-query scan): every query's groups equal the ordinary path's for its own constants, on two
    runs with different constants; other expressions are refused.  Prints the latency of 6 queries run
    one by one against the group."""
    tables = []
    for n, seed in ((1 << 20, 0), (300_001, 1), (2_500_000, 2), (70_000, 3), (1_200_000, 4), (1 << 20, 5)):
        t = W.pricing_summary(n, seed=seed) if kind != "hash" else W.filter_groupby_1m(n, seed=seed)
        t.to_device()
        tables.append(t)
    ops.jit_set_mode(abi.JIT_SYNC)
    exs, group = [], None
    try:
        qs = []
        for t in tables:
            if kind == "hash":
                e, aq = W.filter_groupby_1m_query(t)
                ds, cap, c0 = None, 1024, 500_000
            elif kind == "dense":
                e, aq, ds = W.pricing_summary_query(t)
                cap, c0 = 1024, 2467
            else:
                e = W.env_for(t)
                aq = q.AggQuery(e, q.col(0).le(2467), [],
                                [q.Agg("COUNT"), q.Agg("SUM", q.col(2) * (q.ilit(100) - q.col(3)), "BIGINT", False),
                                 q.Agg("MIN", q.col(2), "BIGINT", True)])
                ds, cap, c0 = None, 1, 2467
            qs.append((t, e, aq, ds, cap, const_index(e.env, c0), E.batch_arrays(t.batches(True))))
        fn = {"hash": abi.JF_GROUPED, "dense": abi.JF_DENSE, "nokeys": abi.JF_NOKEYS}[kind]
        e0, aq0 = qs[0][1], qs[0][2]
        prog = ops.jit_get(e0.env, e0.ncols, aq0.plan, fn, "exec group")
        assert prog
        exs = [ops.Executor(aq.plan, cap, ds, e.env, e.ncols, arrays, prog, 64) for _, e, aq, ds, cap, _, arrays in qs]
        group = ops.ExecGroup(exs, prog)
        if kind == "hash":
            cuts = ([500_000, 1, 999_999, 250_000, 0, 777_777], [3, 600_000, 500_000, 999_999, 120_000, 1])
        else:
            cuts = ([2467, 100, 2556, 1500, 2000, 0], [1, 2467, 800, 2556, 2300, 1200])
        for rnd in cuts:
            for (t, e, aq, ds, cap, ci, arrays), c in zip(qs, rnd):
                set_int_const(e.env, ci, c)
            group.run([e.env for _, e, *_ in qs])
            ops.sync()
            for ex, (t, e, aq, ds, cap, ci, arrays) in zip(exs, qs):
                k, x, st = ex.results()
                ovf, rk, rx = ordinary(aq.plan, cap, ds, e.env, e.ncols, arrays, prog)
                assert not ovf and st["overflow"] == 0 and st["error"] == 0
                assert st["groups"] == rk.shape[0]
                same_groups(aq.plan, k, x, rk, rx)
        # other expressions are refused
        bad = abi.ExprEnv()
        ctypes.memmove(ctypes.addressof(bad), ctypes.addressof(qs[0][1].env), ctypes.sizeof(bad))
        bad.code[0].op = (bad.code[0].op + 1) % 250
        with pytest.raises(ops.WsError) as ei:
            group.run([bad] + [e.env for _, e, *_ in qs[1:]])
        assert ei.value.code == 1210
        # latency: the six queries one by one, against the group
        n = 50

        def alone():
            for ex, (_, e, *_r) in zip(exs, qs):
                ex.run(e.env)
            ops.sync()

        def together():
            group.run([e.env for _, e, *_ in qs])
            ops.sync()

        out = {}
        for name, f in (("one by one", alone), ("group", together)):
            for _ in range(5):
                f()
            t0 = time.perf_counter()
            for _ in range(n):
                f()
            out[name] = (time.perf_counter() - t0) / n * 1e6
        print(f"\n[exec] {kind}: 6 prepared queries " + ", ".join(f"{k} {v:.0f} us" for k, v in out.items()))
    finally:
        if group is not None:
            group.close()
        for ex in exs:
            ex.close()
        ops.jit_set_mode(-1)
        for t in tables:
            t.free_device()


def test_group_refuses_mixed_plans_and_kinds(fg):
    """A group needs one compiled plan and one scan kind with a multi-query form: executors of two
    plans (hash and no-key) are refused before anything is captured, as is an executor given twice."""
    e, aq = W.filter_groupby_1m_query(fg)
    ops.jit_set_mode(abi.JIT_SYNC)
    exs = []
    try:
        arrays = E.batch_arrays(fg.batches(True))
        prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_GROUPED, "exec group")
        exs.append(ops.Executor(aq.plan, 1024, None, e.env, e.ncols, arrays, prog, 64))
        e2 = W.env_for(fg)
        aq2 = q.AggQuery(e2, None, [], [q.Agg("COUNT")])
        prog2 = ops.jit_get(e2.env, e2.ncols, aq2.plan, abi.JF_NOKEYS, "exec group")
        exs.append(ops.Executor(aq2.plan, 1, None, e2.env, e2.ncols, arrays, prog2, 1))
        for members in ([exs[0], exs[1]], [exs[0], exs[0]]):
            with pytest.raises(ops.WsError) as ei:
                ops.ExecGroup(members, prog)
            assert ei.value.code == 1210
        # the executors still run on their own
        exs[0].run(e.env)
        ops.sync()
        _, _, st = exs[0].results()
        assert st["error"] == 0 and st["groups"] > 0
    finally:
        for x in exs:
            x.close()
        ops.jit_set_mode(-1)
