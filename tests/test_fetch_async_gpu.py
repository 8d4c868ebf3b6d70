"""The one-sync fetch (ws_agg_fetch_async): the groups the GPU writes straight into pinned host memory
are the ones ws_agg_fetch returns, word for word and in the same order (dense, hash, multi-key and
no-key plans, with and without the compiled plan), whole or range by range; an overflowed hash run
writes nothing and says so in the status; ordinary host memory is refused."""
import ctypes as C

import numpy as np
import pytest

from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .test_agg_gpu import gpu_aggregate

pytestmark = pytest.mark.gpu


def fetch_async(agg, max_groups, first=0):
    nk, na = agg.plan.nkeys, agg.plan.naggs
    hk = ops.HostBuffer((max(max_groups, 1), max(nk, 1)), np.float64)
    hx = ops.HostBuffer((max(max_groups, 1), na, 2), np.int64)
    st = ops.HostBuffer(1, ops.FETCH_STATUS)
    hk.array.fill(0)
    hx.array.fill(0)
    agg.fetch_async(max_groups, hk if nk else None, hx, st, first)
    ops.sync()
    s = st.array[0]
    g = int(s["groups"])
    m = max(0, min(g - first, max_groups))
    out = (g, int(s["overflow"]), int(s["error"]), hk.array[:m, :nk].copy(), hx.array[:m].copy(), hx.array.copy())
    for b in (hk, hx, st):
        b.close()
    return out


def same_as_fetch(agg):
    keys, _, ex = agg.fetch()
    g, ovf, err, k2, x2, _ = fetch_async(agg, keys.shape[0] + 5)
    assert (g, ovf, err) == (keys.shape[0], 0, 0)
    assert np.array_equal(keys.view(np.int64), k2.view(np.int64))
    assert np.array_equal(ex, x2)


@pytest.mark.parametrize("jit", [True, False], ids=["compiled", "interpreted"])
def test_dense_hash_and_nokeys_equal_fetch(jit):
    t = W.pricing_summary(1_300_000, seed=5)
    e, aq, ds = W.pricing_summary_query(t)
    for dense, cap in ((ds, 1024), (None, 64)):
        agg = gpu_aggregate(t, e, aq.plan, dense, cap, jit)
        same_as_fetch(agg)
        agg.close()
    e2 = W.env_for(t)
    aq2 = q.AggQuery(e2, q.col(0).le(2467), [], [q.Agg("COUNT"), q.Agg("SUM", q.col(2), "BIGINT", True),
                                                   q.Agg("MIN", q.col(2), "BIGINT", True)])
    agg = gpu_aggregate(t, e2, aq2.plan, None, 1024, jit)
    same_as_fetch(agg)
    agg.close()


def test_multi_key_many_groups_equal_fetch():
    n = 900_000
    rng = np.random.default_rng(21)
    t = W.Table(n, seg_rows=1 << 18)
    t.add("a", abi.T_I32, rng.integers(0, 700, n, dtype=np.int32))
    t.add("b", abi.T_I64, rng.integers(-1, 400, n, dtype=np.int64))
    t.add("f", abi.T_F64, np.round(rng.random(n) * 4) / 2 - 1.0)
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True), (q.col(1), True), (q.col(2), False)],
                    [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MAX", q.col(2), "DOUBLE", True)])
    agg = gpu_aggregate(t, e, aq.plan, None, 1 << 21)
    assert not agg.overflowed()
    same_as_fetch(agg)
    agg.close()


def test_overflow_writes_nothing_and_ranges_assemble():
    n = 400_000
    rng = np.random.default_rng(3)
    t = W.Table(n, seg_rows=1 << 17)
    t.add("k", abi.T_I64, rng.integers(0, 50_000, n, dtype=np.int64))
    t.add("v", abi.T_I64, rng.integers(0, 100, n, dtype=np.int64))
    e = W.env_for(t)
    aq = q.AggQuery(e, None, [(q.col(0), True)], [q.Agg("SUM", q.col(1), "BIGINT", True)])
    agg = gpu_aggregate(t, e, aq.plan, None, 1024)
    assert agg.overflowed()
    g, ovf, err, _, _, whole = fetch_async(agg, 1 << 16)
    assert ovf == 1 and err == 0 and not whole.any()
    agg.close()
    agg = gpu_aggregate(t, e, aq.plan, None, 1 << 17)
    keys, _, ex = agg.fetch()
    # range by range (ragged last range, a range past the end): the same groups in the same order
    parts_k, parts_x, first = [], [], 0
    while first <= keys.shape[0]:
        g, ovf, err, k2, x2, _ = fetch_async(agg, 4999, first)
        assert (g, ovf, err) == (keys.shape[0], 0, 0)
        parts_k.append(k2)
        parts_x.append(x2)
        first += 4999
    assert np.array_equal(np.concatenate(parts_k).view(np.int64), keys.view(np.int64))
    assert np.array_equal(np.concatenate(parts_x), ex)
    # ordinary (pageable) host memory is refused
    x = np.zeros((keys.shape[0], aq.plan.naggs, 2), np.int64)
    k = np.zeros((keys.shape[0], 1))
    st = ops.HostBuffer(1, ops.FETCH_STATUS)
    rc = ops.lib().ws_agg_fetch_async(agg.h, 0, keys.shape[0], k.ctypes.data, x.ctypes.data, st.ptr)
    assert rc == 1210
    st.close()
    agg.close()
