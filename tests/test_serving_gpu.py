"""The request loop: every query's result in the mix (overlapping on the device with others) equals
its result alone — integer slots exactly, DOUBLE sums within 1e-12 relative — in both serving forms,
into result arrays and through per-worker buffers (digests); QPS and p50 / p99 of the forms are
printed."""
import numpy as np
import pytest

from warpstore_b200 import abi, ops
from warpstore_b200 import serving as S

from .helpers import DOUBLE_RTOL

pytestmark = pytest.mark.gpu


def same(a_keys, a_ex, b_keys, b_ex):
    ka, kb = np.ascontiguousarray(a_keys).view(np.int64), np.ascontiguousarray(b_keys).view(np.int64)
    oa, ob = np.lexsort(ka.T[::-1]), np.lexsort(kb.T[::-1])
    assert np.array_equal(ka[oa], kb[ob])
    xa, xb = a_ex[oa], b_ex[ob]
    ints = [0, 1, 2, 3, 4]  # COUNT, SUM(v) halves, MIN, MAX: exact
    assert np.array_equal(xa[:, ints], xb[:, ints])
    da, db = xa[:, 5, 0].view(np.float64), xb[:, 5, 0].view(np.float64)
    np.testing.assert_allclose(da, db, rtol=DOUBLE_RTOL, atol=1e-300)


def test_results_alone_equal_results_in_the_mix():
    tables = S.make_tables(8, 10_000, 2_000_000, seed=5)
    for t in tables:
        t.to_device()
    queries = S.make_queries(tables, 160, rate=2000.0, seed=6)
    prepared, arrays = S.prepare(tables, queries)
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        alone = {p.qr.qid: S.run_alone(p, arrays, False) for p in prepared}  # each query by itself
        rows = {q: a[0].shape[0] for q, a in alone.items()}
        S.run_native(tables, prepared, arrays, "batched", result_rows=rows)  # warm: pools, estimator weights
        for loop in ("python", "native"):
            for mode in ("plain", "batched"):
                if loop == "python":
                    st = S.run(tables, prepared, arrays, mode)
                else:
                    st = S.run_native(tables, prepared, arrays, mode, result_rows=rows)
                assert st.completed == len(queries)
                for p in prepared:
                    r = st.results[p.qr.qid]
                    same(*alone[p.qr.qid], r.keys, r.exact)
                print(f"\n[serving] {loop} loop, {mode}: {st.qps:.0f} QPS, p50 {st.p50_ms:.2f} ms, "
                      f"p99 {st.p99_ms:.2f} ms, overflow reruns {st.overflow_reruns}")
        # results delivered to per-worker buffers (pageable / pinned, range by range through a buffer
        # smaller than the largest result) and digested as they arrive: the digests of the results alone
        want = {p.qr.qid: S.digest(p.plan, *alone[p.qr.qid]) for p in prepared}
        big = max(rows.values())
        for mode in ("plain", "batched"):
            st = S.run_native(tables, prepared, arrays, mode, keep_results=False, arena_bytes=big * 40, checksum=True)
            for p in prepared:
                r = st.results[p.qr.qid]
                c, f = want[p.qr.qid]
                assert r.groups == rows[p.qr.qid] and r.checksum == c
                assert abs(r.fsum - f) <= 1e-9 * max(abs(f), 1e-300)
            print(f"\n[serving] native loop, {mode}, results to per-worker buffers: {st.qps:.0f} QPS, "
                  f"p50 {st.p50_ms:.2f} ms, p99 {st.p99_ms:.2f} ms")
        # arrived queries of one plan sharing a scan launch (ws_agg_run_many): compiled plans (queries of
        # the same shape only) and interpreted ones (any queries of the hash kind), all arriving at once
        import dataclasses
        burst = [dataclasses.replace(p, qr=dataclasses.replace(p.qr, arrival=0.0)) for p in prepared]
        interp = [dataclasses.replace(p, prog=None) for p in burst]
        for name, prep in (("compiled", burst), ("interpreted", interp)):
            st = S.run_native(tables, prep, arrays, "batched", result_rows=rows, batch=8)
            assert st.completed == len(queries)
            for p in prep:
                r = st.results[p.qr.qid]
                same(*alone[p.qr.qid], r.keys, r.exact)
            print(f"\n[serving] native loop, batched, {name} plans, up to 8 queries per launch: {st.qps:.0f} QPS")
    finally:
        ops.jit_set_mode(-1)
        for t in tables:
            t.free_device()


def test_a_failing_query_ends_the_loop_with_its_error():
    """A query whose operator call fails (a column count the library refuses) ends ws_serve with that
    query's error code once the workers in flight have finished; nothing hangs and the library stays
    usable for the next call."""
    tables = S.make_tables(2, 10_000, 200_000, seed=7)
    for t in tables:
        t.to_device()
    queries = S.make_queries(tables, 24, rate=5000.0, seed=8)
    prepared, arrays = S.prepare(tables, queries)
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        bad = prepared[5]
        saved = bad.ncols
        bad.ncols = abi.MAX_COLS + 1  # refused by every entry point before any memory is read
        for mode in ("plain", "batched"):
            with pytest.raises(ops.WsError) as ei:
                S.run_native(tables, prepared, arrays, mode, keep_results=False)
            assert ei.value.code == 1210
        bad.ncols = saved
        st = S.run_native(tables, prepared, arrays, "batched", keep_results=False)
        assert st.completed == len(queries)
    finally:
        ops.jit_set_mode(-1)
        for t in tables:
            t.free_device()
