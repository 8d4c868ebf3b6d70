"""Parity with the reference itself: the reference's own GPU operators (Warpstore src/gpu.cu and src/jit.cu
built for sm_100a into oracle/_ref) run on the same device inputs as ours — its compiled plans (the
engine's production path), and for the aggregations and known answers its interpreted kernels too.

Compared in the engine's result format (the reference's fetch): keys, COUNT, integer MIN / MAX and
split BIGINT sums (recombined as the engine does) bit-exact; DOUBLE sums within 1e-12 relative.
Integer-expression sums without aggBits are accumulated by the reference through FP64 atomics
(src/kernels.cuh:499-506) while ours are exact int128: compared within 1e-12 relative, with the exact
value checked against the CPU oracle elsewhere.  Join pairs are compared as sorted multisets,
selections index for index.  Each test prints both operators' times (the reference's own sm_100 build
vs this library)."""
import numpy as np
import pytest

from oracle import ref
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from . import known_answers as KA

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")]


def ours(t, e, aq, dense, cap, fn):
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, fn, "refcmp")
        res = []
        for rep in range(2):  # second run timed (plan compiled, pool warm)
            import torch
            agg = ops.GpuAggregator(aq.plan, cap, dense)
            for s in range(t.nseg):
                for i, v in enumerate(t.views(s, True)):
                    e.env.cols[i] = v
                agg.add_batch(e.env, e.ncols, t.seg_len(s))
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record()
            agg.run(e.env, prog)
            agg.overflowed()
            s1.record()
            s1.synchronize()
            keys, accs, ex = agg.fetch()
            res = (keys, accs, s0.elapsed_time(s1))
            agg.close()
        return res
    finally:
        ops.jit_set_mode(-1)


def by_key(keys, accs):
    kb = np.ascontiguousarray(keys).view(np.int64) if keys.size else np.zeros((accs.shape[0], 0), np.int64)
    order = np.lexsort(kb.T[::-1]) if kb.shape[1] else np.arange(accs.shape[0])
    return kb[order], accs[order]


def compare_engine_format(aq, keys_a, accs_a, keys_b, accs_b, hi_b=None):
    ka, aa = by_key(keys_a, accs_a)
    kb, ab = by_key(keys_b, accs_b)
    assert np.array_equal(ka, kb), "group keys differ"
    plan = aq.plan
    bits_a, bits_b = aa.view(np.int64), ab.view(np.int64)
    for a in aq.aggs:
        s = a.slot
        if a.fn == "COUNT" or s == 0:
            assert np.array_equal(aa[:, s], ab[:, s]), f"{a.fn} slot {s}"
        elif a.hi_slot >= 0 and plan.aggBits[a.hi_slot]:
            wa = bits_a[:, a.hi_slot].astype(object) * (1 << 32) + bits_a[:, s].astype(object)
            wb = bits_b[:, a.hi_slot].astype(object) * (1 << 32) + bits_b[:, s].astype(object)
            assert list(wa) == list(wb), f"split sum slot {s}"
        elif plan.aggBits[s]:
            assert np.array_equal(bits_a[:, s], bits_b[:, s]), f"int64 bits slot {s}"
        else:
            np.testing.assert_allclose(aa[:, s], ab[:, s], rtol=1e-12, err_msg=f"{a.fn} slot {s}")


def ref_aggregate(e, aq, batches, dense, cap, compiled):
    """The reference's aggregation, compiled plan or interpreted; the second run is timed (plan
    compiled, pool warm).  (keys, accs, milliseconds of run() + overflowed())."""
    ref.set_compiled(compiled)
    try:
        for _ in range(2):
            rk, ra, _, ovf, rms = ref.aggregate(e.env, e.ncols, aq.plan, batches, dense, cap)
            assert not ovf
            assert ref.last_compiled() == compiled, "the reference did not run the plan kind asked for"
    finally:
        ref.set_compiled(True)
    return rk, ra, rms


def test_filter_groupby_vs_reference():
    t = W.filter_groupby_1m(1 << 20, seed=0)
    e, aq = W.filter_groupby_1m_query(t)
    t.to_device()
    rk, ra, rms = ref_aggregate(e, aq, t.batches(True), None, 1024, True)
    ik, ia, ims = ref_aggregate(e, aq, t.batches(True), None, 1024, False)
    ok_, oa, oms = ours(t, e, aq, None, 1024, abi.JF_GROUPED)
    compare_engine_format(aq, ok_, oa, rk, ra)
    compare_engine_format(aq, ok_, oa, ik, ia)
    print(f"\n[timing] filter_groupby_1m hash: reference compiled {rms:.3f} ms (interpreted {ims:.3f} ms), "
          f"ours {oms:.3f} ms")


def test_pricing_summary_vs_reference():
    t = W.pricing_summary(8 * W.SEG_ROWS, seed=2)
    e, aq, ds = W.pricing_summary_query(t)
    t.to_device()
    rk, ra, rms = ref_aggregate(e, aq, t.batches(True), ds, 1024, True)
    ik, ia, ims = ref_aggregate(e, aq, t.batches(True), ds, 1024, False)
    ok_, oa, oms = ours(t, e, aq, ds, 1024, abi.JF_DENSE)
    compare_engine_format(aq, ok_, oa, rk, ra)
    compare_engine_format(aq, ok_, oa, ik, ia)
    rows = t.n
    print(f"\n[timing] pricing_summary {rows} rows dense: reference compiled {rms:.3f} ms "
          f"({rows / rms / 1e6:.1f} G rows/s; interpreted {ims:.3f} ms), ours {oms:.3f} ms ({rows / oms / 1e6:.1f} G rows/s)")


def test_join_vs_reference():
    rng = np.random.default_rng(3)
    nb, np_ = 2_000_000, 8_000_000
    bk = rng.permutation(4_000_000)[:nb].astype(np.int64)
    pk = rng.integers(0, 4_000_000, np_).astype(np.int64)
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    bv, pv = abi.ColView(db.ptr, abi.T_I64, 0, 0, 0), abi.ColView(dp.ptr, abi.T_I64, 0, 0, 0)
    rb, rp, rms = ref.hash_join(bv, nb, pv, np_)
    import torch
    for rep in range(2):
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        ob, op, m = ops.hash_join(bv, nb, pv, np_)
        s1.record()
        s1.synchronize()
        oms = s0.elapsed_time(s1)
        gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
        ops.tmp_free(ob)
        ops.tmp_free(op)
    assert m == len(rb)
    g, r = np.lexsort((gb, gp)), np.lexsort((rb, rp))
    assert np.array_equal(gp[g], rp[r]) and np.array_equal(gb[g], rb[r])
    print(f"\n[timing] hash join build {nb} probe {np_}: reference {rms:.3f} ms, ours {oms:.3f} ms")


@pytest.mark.parametrize("nb,np_", [(7_500_000, 60_000_000), (7_500_000, 8_000_000)], ids=["60m", "8m"])
def test_sparse_key_join_vs_reference(nb, np_):
    """Build keys spread over all of int64 (the hash path, no dense range): pairs keyed alike, the
    reference's pair count; CUDA-event times of both (second run)."""
    import torch
    rng = np.random.default_rng(3)
    mul = np.uint64(0x9E3779B97F4A7C15)
    bk = (rng.permutation(15_000_000)[:nb].astype(np.uint64) * mul).view(np.int64)
    pk = (rng.integers(0, 15_000_000, np_).astype(np.uint64) * mul).view(np.int64)
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    bv, pv = abi.ColView(db.ptr, abi.T_I64, 0, 0, 0), abi.ColView(dp.ptr, abi.T_I64, 0, 0, 0)
    times = {}
    for rep in range(2):
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        rb, rp, rm, _ = ref.hash_join_dev(bv, nb, pv, np_)
        s1.record()
        s1.synchronize()
        times["reference"] = s0.elapsed_time(s1)
        ref.free(rb)
        ref.free(rp)
        s0.record()
        ob, op, m = ops.hash_join(bv, nb, pv, np_)
        s1.record()
        s1.synchronize()
        times["ours"] = s0.elapsed_time(s1)
        gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
        ops.tmp_free(ob)
        ops.tmp_free(op)
    assert m == rm and m > 0
    assert np.array_equal(bk[gb], pk[gp])            # every pair's keys are equal
    assert np.unique(gp).size == m                   # unique build keys: one pair per matching probe row
    print(f"\n[timing] sparse-key hash join build {nb} probe {np_}: reference {times['reference']:.3f} ms, "
          f"ours {times['ours']:.3f} ms")


def test_select_vs_reference():
    t = W.pricing_summary(3 * W.SEG_ROWS + 12345, seed=4)
    e = W.env_for(t)
    where = e.compile(q.and_(q.col(0).lt(1203), q.col(3).ge(5)))
    t.to_device()
    ri, rp = ref.select_multi(e.env, where, t.batches(True), e.ncols)
    assert ref.last_compiled()
    ptr, m, per = ops.select_multi(e.env, where, t.batches(True), e.ncols)
    gi = ops.device_to_array(ptr, np.int32, m)
    ops.tmp_free(ptr)
    assert np.array_equal(gi, ri) and list(per) == list(rp)


@pytest.mark.parametrize("compiled", [True, False], ids=["compiled", "interpreted"])
@pytest.mark.parametrize("case", KA.load()["cases"], ids=lambda c: c["name"])
def test_known_answers_on_reference(case, compiled):
    """The harness itself reproduces the reference's known answers (tests/smoke.py) on the GPU, with its
    compiled plans and with its interpreter."""
    g = KA.load()
    st = g["states"][str(case["state"])]
    t = KA.table_of(st)
    t.to_device()
    bset = ops.DeviceBuffer.from_array(np.array([0b0010], dtype=np.uint32))
    e, aq, post = KA.plan_of(case, t, bset.ptr)
    bits = KA.deleted_bits(st)
    dbits = ops.DeviceBuffer.from_array(bits) if bits is not None else None
    ref.set_compiled(compiled)
    try:
        rk, ra, hi, ovf, _ = ref.aggregate(e.env, e.ncols, aq.plan, [(t.n, dbits.ptr if dbits else 0, t.views(0, True))])
        assert ref.last_compiled() == compiled
    finally:
        ref.set_compiled(True)
    assert not ovf
    agg_rows = []
    rkb = rk.view(np.int64) if rk.size else np.zeros((ra.shape[0], 0), np.int64)
    for gi in range(ra.shape[0]):
        row = [int(x) for x in rkb[gi]]
        for a in aq.aggs:
            v = ra[gi, a.slot]
            if a.fn == "COUNT" or a.arg_type != "DOUBLE":
                if aq.plan.nkeys == 0 and aq.plan.aggInt[a.slot] and a.fn != "COUNT":
                    v = float(ra[gi:gi + 1, a.slot].view(np.int64)[0])
                row.append(int(v))
            else:
                row.append(float(v))
        agg_rows.append(row)
    if post:
        agg_rows = [r for r in agg_rows if post(r)]
    agg_rows.sort(key=(lambda r: -r[1]) if case["name"] == "having" else None)
    assert agg_rows == case["expect"]
