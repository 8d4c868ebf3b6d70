"""The CPU oracle pinned against the reference's known answers (tests/golden/known_answers.json, from
the reference's tests/smoke.py) and against brute-force numpy on the benchmark workloads."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from . import known_answers as KA


@pytest.mark.parametrize("case", KA.load()["cases"], ids=lambda c: c["name"])
def test_known_answers(built, case):
    g = KA.load()
    st = g["states"][str(case["state"])]
    t = KA.table_of(st)
    bset = np.array([0b0010], dtype=np.uint32)  # LIKE 'b%': banana (code 1)
    e, aq, post = KA.plan_of(case, t, bset.ctypes.data)
    bits = KA.deleted_bits(st)
    keys, words, ovf = oracle.aggregate(e.env, aq.plan, t.batches(False, [bits.ctypes.data] if bits is not None else None),
                                        e.ncols, nthreads=2)
    assert not ovf
    assert KA.result_rows(case, aq, keys, words, post) == case["expect"]


def test_pricing_summary_brute_force(built):
    n = 300_000
    t = W.pricing_summary(n, seed=5)
    e, aq, ds = W.pricing_summary_query(t)
    keys, words, ovf = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols, nthreads=4)
    sd, qty, price, disc, tax, f1, f2 = (c.data.astype(object) if i in (1, 2, 3, 4) else c.data for i, c in enumerate(t.cols))
    m = t.cols[0].data <= 2467
    f1v, f2v = t.cols[5].data, t.cols[6].data
    for gi, (k1, k2) in enumerate(keys):
        sel = m & (f1v == k1) & (f2v == k2)
        assert words[gi, 0, 0] == sel.sum()
        dp = price[sel] * (100 - disc[sel])
        ch = dp * (100 + tax[sel])
        sums = {aq.aggs[1].slot: qty[sel].sum(), aq.aggs[2].slot: price[sel].sum(), aq.aggs[3].slot: dp.sum(),
                aq.aggs[4].slot: ch.sum()}
        for slot, want in sums.items():
            lo, hi = words[gi, slot]
            assert int(np.uint64(lo)) + (int(hi) << 64) == int(want)


def test_filter_groupby_brute_force(built):
    t = W.filter_groupby_1m(200_000, seed=3)
    e, aq = W.filter_groupby_1m_query(t)
    keys, words, _ = oracle.aggregate(e.env, aq.plan, t.batches(False), e.ncols, nthreads=3)
    k, v, f = (c.data for c in t.cols)
    m = v < 500_000
    assert keys.shape[0] == len(np.unique(k[m]))
    for gi, kk in enumerate(keys[:, 0]):
        s = m & (k == kk)
        assert words[gi, 0, 0] == s.sum()
        assert words[gi, aq.aggs[1].slot, 0] == v[s].sum()
        assert words[gi, aq.aggs[2].slot, 0] == v[s].min() and words[gi, aq.aggs[3].slot, 0] == v[s].max()
        fs = words[gi, aq.aggs[4].slot, 0:1].view(np.float64)[0]
        assert abs(fs - f[s].sum()) <= 1e-12 * abs(f[s].sum())


def test_three_valued_logic_and_overflow(built):
    t = W.Table(4)
    t.add("a", abi.T_I64N, np.array([1, abi.NULL_I64, 3, 2**62], dtype=np.int64))
    t.add("b", abi.T_I64, np.array([0, 5, -1, 2**62], dtype=np.int64))
    e = W.env_for(t)
    views = t.views(0, False)
    cases = [
        (q.or_(q.col(0).gt(0), q.col(1).gt(100)), [1.0, None, 1.0, 1.0]),      # NULL OR false = NULL
        (q.and_(q.col(0).gt(0), q.col(1).lt(0)), [0.0, 0.0, 1.0, 0.0]),        # NULL AND false = false
        (q.coalesce(q.col(0), q.lit(7.0)), [1.0, 7.0, 3.0, float(2**62)]),
        (q.col(1) / q.ilit(0), [None] * 4),                                  # x / 0 = NULL
    ]
    for ex, want in cases:
        p = e.compile(ex)
        for r, w in enumerate(want):
            d, iv, isint, ovf = oracle.eval_row(e.env, views, p, r)
            assert (d != d) if w is None else d == w
    p = e.compile(q.col(1) * q.ilit(4))
    assert oracle.eval_row(e.env, views, p, 3)[3]          # 2^62 * 4 overflows int64: flagged
    assert not oracle.eval_row(e.env, views, p, 2)[3]


def test_dates_match_python(built):
    import datetime
    rng = np.random.default_rng(0)
    dd = rng.integers(-50000, 80000, 200).astype(np.int32)
    t = W.Table(len(dd))
    t.add("d", abi.T_I32, dd)
    e = W.env_for(t)
    views = t.views(0, False)
    fns = {"MONTH": lambda x: x.month, "DAY": lambda x: x.day, "DAYOFYEAR": lambda x: x.timetuple().tm_yday,
           "QUARTER": lambda x: (x.month - 1) // 3 + 1, "WEEKDAY": lambda x: x.weekday(),
           "DAYOFWEEK": lambda x: (x.isoweekday() % 7) + 1}
    progs = {k: e.compile(q.call1(k, q.col(0))) for k in fns}
    py = e.compile(q.year(q.col(0)))
    for r, x in enumerate(dd):
        date = datetime.date(1970, 1, 1) + datetime.timedelta(days=int(x))
        assert oracle.eval_row(e.env, views, py, r)[1] == date.year
        for k, f in fns.items():
            assert oracle.eval_row(e.env, views, progs[k], r)[0] == f(date), (k, date)


@pytest.mark.parametrize("enc", [7, 8], ids=["bitpack", "rle"])
def test_bitpack_and_rle_segments_decode(enc):
    """The library's integer segment formats (enc 7 bit-packed, enc 8 run-length): every stored row
    decodes to its value, NULLs included, across several segments."""
    rng = np.random.default_rng(enc)
    n = 50_003
    a = rng.integers(-10**6, 10**6, n).astype(np.int64)
    a[rng.random(n) < 0.1] = abi.NULL_I64
    r = np.repeat(rng.integers(0, 100, n // 40 + 1), 40)[:n].astype(np.int32)
    r[rng.random(n) < 0.01] = abi.NULL_I32
    t = W.Table(n, seg_rows=1 << 13)
    t.add("a", abi.T_I64N, a, enc=enc)
    t.add("r", abi.T_I32N, r, enc=enc)
    e = W.env_for(t)
    progs = [e.compile(q.col(0)), e.compile(q.col(1))]
    for s in range(t.nseg):
        vs = t.views(s, False)
        lo = s * t.seg_rows
        for row in rng.integers(0, t.seg_len(s), 40):
            for c, src, nul in ((0, a, abi.NULL_I64), (1, r, abi.NULL_I32)):
                d, _, _, _ = oracle.eval_row(e.env, vs, progs[c], int(row))
                want = src[lo + row]
                assert (d != d) == (want == nul)
                assert d != d or d == float(want)
