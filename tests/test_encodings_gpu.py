"""Bit-packed (enc 7) and run-length (enc 8) integer segments on the GPU: scans over them (filter +
dense / hash GROUP BY, compiled and interpreted; selection; gathers; range-scan offsets) give the same
results as over the raw columns and as the CPU oracle, and the GPU segment encoder writes exactly the
bytes of the host encoder."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .helpers import compare_exact

pytestmark = pytest.mark.gpu


def tables(enc, n=300_001, seed=11):
    """The same data raw and with every integer column in `enc`."""
    rng = np.random.default_rng(seed)
    k = np.repeat(rng.integers(0, 12, n // 64 + 1), 64)[:n].astype(np.int32)   # long runs: RLE-friendly
    v = rng.integers(-50_000, 50_000, n).astype(np.int64)
    v[rng.random(n) < 0.05] = abi.NULL_I64
    d = rng.integers(0, 2_000, n).astype(np.int32)
    out = []
    for e in (0, enc):
        t = W.Table(n, seg_rows=1 << 16)
        t.add("k", abi.T_I32, k, enc=e)
        t.add("v", abi.T_I64N, v, enc=e)
        t.add("d", abi.T_I32, d, enc=e)
        out.append(t)
    return out


def run_agg(t, e, aq, jit, ds=None):
    t.to_device()
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        fn = abi.JF_DENSE if ds is not None else abi.JF_GROUPED
        prog = ops.jit_get(e.env, e.ncols, aq.plan, fn, "enc") if jit else None
        agg = ops.GpuAggregator(aq.plan, 1 << 12, ds)
        agg.add_batches(e.ncols, t.batches(True))
        agg.run(e.env, prog)
        assert not agg.overflowed()
        keys, _, ex = agg.fetch()
        agg.close()
        return keys, ex
    finally:
        ops.jit_set_mode(-1)


@pytest.mark.parametrize("jit", [True, False], ids=["compiled", "interpreted"])
@pytest.mark.parametrize("enc", [7, 8], ids=["bitpack", "rle"])
@pytest.mark.parametrize("dense", [False, True], ids=["hash", "dense"])
def test_groupby_over_encoded_segments(enc, jit, dense):
    raw, coded = tables(enc)
    results = []
    for t in (raw, coded):
        e = W.env_for(t)
        aq = q.AggQuery(e, q.col(2).lt(1500), [(q.col(0), True)],
                        [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True), q.Agg("MIN", q.col(1), "BIGINT", True),
                         q.Agg("MAX", q.col(2), "INT", True), q.Agg("SUM", q.col(1) * q.col(2), "BIGINT", False)])
        ds = q.dense_spec(aq.plan, [(0, 11)], t.n) if dense else None
        results.append(run_agg(t, e, aq, jit, ds))
        if t is coded:
            ok, ow, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols)
            compare_exact(aq.plan, results[-1][0], results[-1][1], ok, ow)
        t.free_device()
    (rk, rx), (ck, cx) = results
    assert np.array_equal(rk.view(np.int64), ck.view(np.int64)) and np.array_equal(rx, cx)


@pytest.mark.parametrize("enc", [7, 8], ids=["bitpack", "rle"])
def test_select_and_gather_over_encoded_segments(enc):
    raw, coded = tables(enc, seed=12)
    for t in (raw, coded):
        t.to_device()
    e = W.env_for(coded)
    where = e.compile(q.and_(q.col(1).ge(0), q.col(0).lt(6)))
    ri = ops.select_multi(e.env, where, raw.batches(True), e.ncols)
    ci = ops.select_multi(e.env, where, coded.batches(True), e.ncols)
    a = ops.device_to_array(ri[0], np.int32, ri[1])
    b = ops.device_to_array(ci[0], np.int32, ci[1])
    assert np.array_equal(a, b) and list(ri[2]) == list(ci[2])
    boff = [s * coded.seg_rows for s in range(coded.nseg)] + [coded.n]
    for c, pt, dt in ((0, abi.PT_I32, np.int32), (1, abi.PT_I64, np.int64)):
        dst = ops.DeviceBuffer(max(ci[1], 1) * 8)
        ops.gather_multi([coded.views(s, True)[c] for s in range(coded.nseg)], boff[:-1], pt, dt().itemsize, ci[0],
                         ci[1], dst.ptr)
        assert np.array_equal(dst.to_array(dt, ci[1]), coded.cols[c].data[b])
    for p in (ri[0], ci[0]):
        ops.tmp_free(p)
    # a range scan: view offset into a segment
    v = coded.views(1, True)[1]
    v.off = 1234
    idx = np.arange(0, 5_000, 7, dtype=np.int32)
    di = ops.DeviceBuffer.from_array(idx)
    dst = ops.DeviceBuffer(idx.size * 8)
    ops.gather_enc(v, abi.PT_I64, di.ptr, idx.size, dst.ptr)
    assert np.array_equal(dst.to_array(np.int64, idx.size), coded.cols[1].data[coded.seg_rows + 1234 + idx])
    for t in (raw, coded):
        t.free_device()


@pytest.mark.parametrize("enc", [7, 8, 0], ids=["bitpack", "rle", "auto"])
@pytest.mark.parametrize("t,dt,nul", [(abi.T_I32, np.int32, None), (abi.T_I64N, np.int64, abi.NULL_I64),
                                      (abi.T_I32N, np.int32, abi.NULL_I32)])
def test_gpu_encoder_matches_host_encoder(enc, t, dt, nul):
    rng = np.random.default_rng(enc * 10 + t)
    for n, runs in ((1, 1), (1000, 7), (250_001, 4000)):
        x = np.repeat(rng.integers(-3000, 90_000, runs), n // runs + 1)[:n].astype(dt)
        if nul is not None:
            x[rng.random(n) < 0.02] = nul
        d = ops.DeviceBuffer.from_array(x)
        ptr, nbytes, used = ops.encode_column(d.ptr, t, n, enc)
        got = ops.device_to_array(ptr, np.uint8, nbytes)
        ops.tmp_free(ptr)
        want7 = W.encode_bitpack(x, nul)
        want8 = W.encode_rle(x)
        if enc:
            assert used == enc
        else:
            assert used == (8 if want8.size < want7.size else 7)
        assert np.array_equal(got, want7 if used == 7 else want8)


def test_gpu_encoder_rejects_wide_bitpack():
    x = np.array([0, 1 << 40], dtype=np.int64)
    d = ops.DeviceBuffer.from_array(x)
    with pytest.raises(ops.WsError) as ei:
        ops.encode_column(d.ptr, abi.T_I64, 2, 7)
    assert ei.value.code == 1264
    ptr, nbytes, used = ops.encode_column(d.ptr, abi.T_I64, 2, 0)  # auto: run-length
    assert used == 8
    ops.tmp_free(ptr)
