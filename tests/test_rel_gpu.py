"""Parity of the relational helpers with the CPU oracle / numpy: outer and cross joins, join-filter key
bitmaps, deleted bits, code remaps, NULL-aware and encoded gathers, evaluation at rows, the stable
multi-key sort permutation, and an ORDER BY ... LIMIT over compacted groups composed from them as the
engine's post-aggregation does (src/engine_select.cpp:1239-1373)."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

pytestmark = pytest.mark.gpu

NAN = float("nan")


def dev(a):
    return ops.DeviceBuffer.from_array(np.ascontiguousarray(a))


def pairs(ob_ptr, op_ptr, m):
    gb, gp = ops.device_to_array(ob_ptr, np.int32, m), ops.device_to_array(op_ptr, np.int32, m)
    ops.tmp_free(ob_ptr)
    ops.tmp_free(op_ptr)
    return gb, gp


def same_multiset(gb, gp, wb, wp):
    assert len(gb) == len(wb)
    g, w = np.lexsort((gb, gp)), np.lexsort((wb, wp))
    assert np.array_equal(gp[g], wp[w]) and np.array_equal(gb[g], wb[w])


def keys_case(nb, np_, space, seed, dup, nulls, sparse):
    rng = np.random.default_rng(seed)
    bk = rng.integers(0, space, nb) if dup else rng.permutation(max(space, nb))[:nb]
    pk = rng.integers(0, space + space // 4 + 1, np_)  # some probe keys outside the build range
    bk, pk = bk.astype(np.int64), pk.astype(np.int64)
    if sparse:
        mul = np.uint64(0x9E3779B97F4A7C15)
        bk, pk = (bk.astype(np.uint64) * mul).view(np.int64), (pk.astype(np.uint64) * mul).view(np.int64)
    bk[bk == abi.NULL_I64] += 1
    pk[pk == abi.NULL_I64] += 1
    if nulls:
        bk[rng.random(nb) < 0.05] = abi.NULL_I64
        pk[rng.random(np_) < 0.05] = abi.NULL_I64
    return bk, pk


@pytest.mark.parametrize("full", [False, True], ids=["left", "full"])
@pytest.mark.parametrize("sparse", [False, True], ids=["dense-range", "hash"])
@pytest.mark.parametrize("nb,np_,space,dup,nulls", [
    (20_000, 100_000, 30_000, False, False),
    (10_000, 50_000, 3_000, True, True),
    (1, 5, 1, False, False),
])
def test_outer_join(nb, np_, space, dup, nulls, sparse, full):
    bk, pk = keys_case(nb, np_, space, nb + np_ + int(full), dup, nulls, sparse)
    db, dp = dev(bk), dev(pk)
    bv, pv = abi.ColView(db.ptr, abi.T_I64N, 0, 0, 0), abi.ColView(dp.ptr, abi.T_I64N, 0, 0, 0)
    gb, gp = pairs(*ops.hash_join_outer(bv, nb, pv, np_, full))
    wb, wp = oracle.hash_join_outer(abi.ColView(bk.ctypes.data, abi.T_I64N, 0, 0, 0), nb,
                                    abi.ColView(pk.ctypes.data, abi.T_I64N, 0, 0, 0), np_, full)
    same_multiset(gb, gp, wb, wp)
    assert np.array_equal(np.unique(gp[gp >= 0]), np.arange(np_))  # every probe row appears


@pytest.mark.parametrize("full", [False, True], ids=["left", "full"])
def test_outer_join_empty_and_all_null_build(full):
    pk = np.arange(10, dtype=np.int64)
    bk = np.full(7, abi.NULL_I64, dtype=np.int64)
    db, dp = dev(bk), dev(pk)
    for nb in (0, 7):
        gb, gp = pairs(*ops.hash_join_outer(abi.ColView(db.ptr, abi.T_I64N, 0, 0, 0), nb,
                                            abi.ColView(dp.ptr, abi.T_I64N, 0, 0, 0), 10, full))
        wb, wp = oracle.hash_join_outer(abi.ColView(bk.ctypes.data, abi.T_I64N, 0, 0, 0), nb,
                                        abi.ColView(pk.ctypes.data, abi.T_I64N, 0, 0, 0), 10, full)
        same_multiset(gb, gp, wb, wp)


def test_cross_join():
    a, b, m = ops.cross_join(123, 45)
    ga, gb = pairs(a, b, m)
    assert m == 123 * 45
    assert np.array_equal(ga, np.repeat(np.arange(123), 45)) and np.array_equal(gb, np.tile(np.arange(45), 123))
    with pytest.raises(ops.WsError) as ei:
        ops.cross_join(20_000, 20_000)
    assert ei.value.code == 1105


def test_key_bitmap_and_set_bits():
    rng = np.random.default_rng(1)
    k = rng.integers(-500, 5_000, 100_000).astype(np.int32)
    k[rng.random(k.size) < 0.1] = abi.NULL_I32
    dk = dev(k)
    lo, nbits = 100, 3_000
    bits = ops.DeviceBuffer(((nbits + 31) // 32) * 4)
    ops.key_bitmap(abi.ColView(dk.ptr, abi.T_I32N, 0, 0, 0), k.size, lo, nbits, bits.ptr)
    got = np.unpackbits(bits.to_array(np.uint32).view(np.uint8), bitorder="little")[:nbits]
    want = np.zeros(nbits, np.uint8)
    v = k[k != abi.NULL_I32].astype(np.int64) - lo
    want[v[(v >= 0) & (v < nbits)]] = 1
    assert np.array_equal(got, want)
    idx = rng.choice(50_000, 7_000, replace=False).astype(np.int32)
    di = dev(idx)
    dbits = dev(np.zeros(50_000 // 32 + 1, np.uint32))
    ops.set_bits(dbits.ptr, di.ptr, idx.size)
    got = np.unpackbits(dbits.to_array(np.uint32).view(np.uint8), bitorder="little")[:50_000]
    want = np.zeros(50_000, np.uint8)
    want[idx] = 1
    assert np.array_equal(got, want)


def test_remap_bits_gathers():
    rng = np.random.default_rng(2)
    codes = rng.integers(-3, 1_200, 50_000).astype(np.int32)
    codes[rng.random(codes.size) < 0.05] = abi.NULL_I32
    cmap = rng.permutation(1_000).astype(np.int32)
    dc, dm, do = dev(codes), dev(cmap), ops.DeviceBuffer(codes.size * 4)
    ops.remap_codes(dc.ptr, codes.size, dm.ptr, cmap.size, do.ptr)
    want = np.where(codes == abi.NULL_I32, abi.NULL_I32,
                    np.where((codes >= 0) & (codes < cmap.size), cmap[np.clip(codes, 0, cmap.size - 1)], -2))
    assert np.array_equal(do.to_array(np.int32), want)

    ints = rng.integers(-2**62, 2**62, 10_000).astype(np.int64)
    dsrc, ddst = dev(ints.view(np.float64)), ops.DeviceBuffer(ints.size * 8)
    ops.bits_to_double(dsrc.ptr, ints.size, ddst.ptr)
    assert np.array_equal(ddst.to_array(np.float64), ints.astype(np.float64))

    idx = rng.integers(-1, 10_000, 30_000).astype(np.int32)
    di = dev(idx)
    for dt, pt, nul in ((np.int32, abi.PT_I32, abi.NULL_I32), (np.int64, abi.PT_I64, abi.NULL_I64),
                        (np.float64, abi.PT_F64, None)):
        src = (rng.random(10_000) * 1e6).astype(dt)
        ds, dd = dev(src), ops.DeviceBuffer(idx.size * 8)
        ops.gather_null(ds.ptr, pt, di.ptr, idx.size, dd.ptr)
        got = dd.to_array(dt, idx.size)
        want = src[np.clip(idx, 0, None)]
        if nul is None:
            assert np.all(np.isnan(got[idx < 0])) and np.array_equal(got[idx >= 0], want[idx >= 0])
        else:
            assert np.array_equal(got, np.where(idx < 0, nul, want))
    vec = rng.random((10_000, 6)).astype(np.float32)
    dv, dd = dev(vec), ops.DeviceBuffer(idx.size * 24)
    ops.gather_bytes(dv.ptr, 24, di.ptr, idx.size, dd.ptr, True)
    got = dd.to_array(np.float32, idx.size * 6).reshape(-1, 6)
    assert np.array_equal(got[idx >= 0], vec[idx[idx >= 0]])
    assert np.all(np.isnan(got[idx < 0]))  # a NULL vector: every element NaN


def test_gather_encoded_columns():
    rng = np.random.default_rng(3)
    t = W.Table(200_000, seg_rows=200_000)
    t.add("a", abi.T_I32N, np.where(rng.random(200_000) < 0.1, abi.NULL_I32,
                                    rng.integers(1000, 1200, 200_000)).astype(np.int32), enc=1)
    t.add("b", abi.T_I64, rng.integers(-70_000, 0, 200_000).astype(np.int64), enc=3)
    t.to_device()
    idx = rng.integers(0, 200_000, 40_000).astype(np.int32)
    di = dev(idx)
    for c, pt, dt in ((0, abi.PT_I32, np.int32), (1, abi.PT_I64, np.int64)):
        dd = ops.DeviceBuffer(idx.size * 8)
        ops.gather_enc(t.views(0, True)[c], pt, di.ptr, idx.size, dd.ptr)
        assert np.array_equal(dd.to_array(dt, idx.size), t.cols[c].data[idx])
    t.free_device()


@pytest.mark.parametrize("with_idx", [False, True], ids=["rows", "indices"])
def test_eval_at(with_idx):
    rng = np.random.default_rng(4)
    n = 100_000
    t = W.Table(n, seg_rows=n)
    t.add("a", abi.T_I64, rng.integers(-10**6, 10**6, n).astype(np.int64))
    t.add("b", abi.T_I32N, np.where(rng.random(n) < 0.1, abi.NULL_I32, rng.integers(-50, 50, n)).astype(np.int32))
    t.add("f", abi.T_F64, rng.random(n) * 100 - 50)
    t.to_device()
    e = W.env_for(t)
    for i, v in enumerate(t.views(0, True)):
        e.env.cols[i] = v
    idx = rng.integers(0, n, 30_000).astype(np.int32) if with_idx else None
    m = idx.size if with_idx else n
    di = dev(idx) if with_idx else None
    for expr in (q.col(0), q.col(1), q.col(0) * q.ilit(3) - q.col(1), q.col(2) * q.col(0) + q.lit(0.25),
                 q.col(1).lt(10), q.col(0) * q.ilit(7)):
        prog = e.compile(expr)
        for as_int in (False, True):
            out = ops.DeviceBuffer(max(m, 1) * 8)
            (ops.eval_at_int if as_int else ops.eval_at)(e.env, e.ncols, prog, di.ptr if di else None, m, out.ptr)
            got = out.to_array(np.int64 if as_int else np.float64, m)
            want, _ = oracle.eval_at(e.env, t.views(0, False), prog, idx, m, as_int)
            if as_int:
                assert np.array_equal(got, want), expr.canon
            else:
                assert np.array_equal(np.isnan(got), np.isnan(want)), expr.canon
                ok = ~np.isnan(want)
                np.testing.assert_allclose(got[ok], want[ok], rtol=1e-15, err_msg=expr.canon)
    t.free_device()


@pytest.mark.parametrize("m", [1, 1000, 300_001])
def test_sort_perm_matches_stable_sort(m):
    rng = np.random.default_rng(m)
    k0 = rng.integers(0, 5, m).astype(np.float64)  # many ties: stability matters
    k0[rng.random(m) < 0.05] = NAN
    k1 = rng.normal(0, 1e3, m)
    k1[rng.random(m) < 0.1] = 0.0
    k1[rng.random(m) < 0.1] = -0.0
    k1[rng.random(m) < 0.02] = NAN
    k2 = rng.integers(-3, 3, m).astype(np.float64)
    for keys, desc in (([k0], [0]), ([k0], [1]), ([k0, k1], [1, 0]), ([k2, k0, k1], [0, 1, 1])):
        bufs = [dev(k) for k in keys]
        p = ops.sort_perm([b.ptr for b in bufs], desc, m)
        got = ops.device_to_array(p, np.int32, m)
        ops.tmp_free(p)
        assert np.array_equal(got, oracle.sort_perm(keys, desc))


def test_map_rank():
    rng = np.random.default_rng(5)
    rank = rng.permutation(1000).astype(np.int32)
    keys = rng.integers(0, 1000, 20_000).astype(np.float64)
    keys[rng.random(keys.size) < 0.1] = NAN
    dk, dr = dev(keys), dev(rank)
    ops.map_rank(dk.ptr, dr.ptr, keys.size)
    want = np.where(np.isnan(keys), -1.0, rank[np.nan_to_num(keys).astype(np.int64)].astype(np.float64))
    assert np.array_equal(dk.to_array(np.float64), want)


def test_order_by_limit_over_compacted_groups():
    """GROUP BY k ... ORDER BY SUM(v) DESC, k LIMIT 25 on the device: aggregate, compact, the sort keys
    as doubles (exact int64 sums converted), sort permutation, gather of the first 25 groups."""
    t = W.filter_groupby_1m(1 << 20, seed=7)
    e, aq = W.filter_groupby_1m_query(t)
    t.to_device()
    agg = ops.GpuAggregator(aq.plan, 1024)
    for s in range(t.nseg):
        for i, v in enumerate(t.views(s, True)):
            e.env.cols[i] = v
        agg.add_batch(e.env, e.ncols, t.seg_len(s))
    agg.run(e.env, None)
    kp, ap, g = agg.compact()
    a_sum = aq.aggs[1]
    sum_col = ap + a_sum.slot * g * 8
    key_d = ops.DeviceBuffer(g * 8)
    ops.bits_to_double(kp, g, key_d.ptr)  # integer keys are int64 bits
    sum_d = ops.DeviceBuffer(g * 8)
    if aq.plan.aggBits[a_sum.slot]:
        ops.bits_to_double(sum_col, g, sum_d.ptr)
    else:
        sum_d = None
    perm = ops.sort_perm([sum_d.ptr if sum_d else sum_col, key_d.ptr], [1, 0], g)
    top = min(25, g)
    sel = ops.DeviceBuffer(top * 8)
    ops.gather(key_d.ptr, abi.PT_F64, perm, top, sel.ptr)
    got = sel.to_array(np.float64, top)
    keys, accs, _ = agg.fetch(exact=False)
    kk = np.ascontiguousarray(keys[:, 0]).view(np.int64).astype(np.float64)  # integer keys come as int64 bits
    sums = accs[:, a_sum.slot] if not aq.plan.aggBits[a_sum.slot] else accs[:, a_sum.slot].view(np.int64)
    order = oracle.sort_perm([np.asarray(sums, np.float64), kk], [1, 0])
    assert np.array_equal(got, kk[order][:top])
    for p in (kp, ap, perm):
        ops.tmp_free(p)
    agg.close()
    t.free_device()
