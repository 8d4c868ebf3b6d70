"""The estimator on the CPU: the HyperLogLog definition against exact distinct counts; each stored BF16
model against fresh synthetic tables, where it must match the plain estimate at the median and cut its
tail errors (group counts, filter selectivity, join pairs); the zone-map and range-term helpers on
known cases; the dense-vs-hash choice."""
import numpy as np
import pytest

from warpstore_b200 import abi
from warpstore_b200 import estimator as E
from warpstore_b200 import query as q
from warpstore_b200 import train_estimator as T


def test_hll_estimate_accuracy():
    rng = np.random.default_rng(0)
    for k in (10, 1_000, 100_000, 2_000_000):
        keys = rng.integers(0, 1 << 62, k).astype(np.uint64)
        est = E.hll_estimate(E.hll_registers(np.concatenate([keys, keys[: k // 2]])))
        assert abs(est - k) / k < 0.05, (k, est)


def fresh(target, n, seed):
    rng = np.random.default_rng(seed)  # tables the models have not seen (training seeds 0, 1000, 2000)
    if target == "groups":
        data = [T.make_example(rng, None, max_log2_rows=21) for _ in range(n)]  # small: the CPU suite stays quick
    elif target == "rows":
        data = [T.make_rows_example(rng, None, max_log2_rows=21) for _ in range(n)]
    else:
        data = [T.make_pairs_example(rng, max_log2_rows=21) for _ in range(n)]
    return np.stack([d[0] for d in data]), np.array([d[1] for d in data])


@pytest.mark.parametrize("target,n", [("groups", 40), ("rows", 60), ("pairs", 60)])
def test_model_matches_plain_median_and_cuts_tail(target, n):
    m = E.Model(target=target)
    xs, ys = fresh(target, n, 123)
    assert xs.shape[1] == m.nfeatures
    fl = E.FLOOR_LOG2  # capacities start at 1024: counts below are the same to them
    err = np.abs(m.predict_log2_np(xs) - np.maximum(ys, fl))
    plain = np.abs(np.maximum(xs[:, -1], fl) - np.maximum(ys, fl))
    print(f"\n[{target}] |log2 error| median {np.median(err):.3f} p90 {np.quantile(err, 0.9):.3f}; "
          f"plain median {np.median(plain):.3f} p90 {np.quantile(plain, 0.9):.3f}")
    # sizing cares about the tail (an underestimate reruns, an overestimate holds memory): the model
    # must not lose the plain estimate's median and must not widen its tail
    assert np.median(err) <= np.median(plain) + 0.05
    assert np.quantile(err, 0.9) <= np.quantile(plain, 0.9) + 1e-6


def test_features_and_bf16_rounding():
    regs = E.hll_registers(np.arange(5000, dtype=np.uint64))
    x = E.features(regs, 10_000, 5_000, 1_000_000, 1e6)
    assert x.shape == (E.NFEATURES,) and np.all(np.isfinite(x))
    a = np.array([1.0, -2.5, 3.14159, 1e-8, 65504.0], dtype=np.float32)
    r = E.from_bf16(E.to_bf16(a))
    assert np.all(np.abs(r - a) <= np.abs(a) * 2 ** -8)


def test_range_terms():
    where = q.and_(q.and_(q.col(0).lt(5), q.ilit(3).le(q.col(1))), q.col(2).eq(q.col(1)))
    terms, opaque = E.range_terms(where)
    assert sorted(terms) == sorted([(0, abi.OP_LT, 5.0), (1, abi.OP_GE, 3.0)]) and opaque == 1
    assert E.range_terms(None) == ([], 0)
    assert E.range_terms(q.or_(q.col(0).lt(1), q.col(0).gt(9))) == ([], 1)


def test_zone_fractions():
    # segments of 100 rows over [0, 99], [100, 199], [200, 299]; x < 150
    mm = {0: [(0, 99), (100, 199), (200, 299)]}
    lo, est, hi, straddle = E.zone_fractions([(0, abi.OP_LT, 150.0)], 0, [100, 100, 100], mm)
    assert lo == pytest.approx(1 / 3) and hi == pytest.approx(2 / 3) and straddle == pytest.approx(1 / 3)
    assert est == pytest.approx((100 + 100 * 50 / 99) / 300)
    # no statistics for the column: nothing is decided
    lo, est, hi, straddle = E.zone_fractions([(1, abi.OP_LT, 150.0)], 0, [100, 100, 100], mm)
    assert (lo, hi, straddle) == (0.0, 1.0, 1.0)
    # an opaque term: no segment passes entirely
    lo, _, hi, _ = E.zone_fractions([(0, abi.OP_GE, 0.0)], 1, [100, 100, 100], mm)
    assert lo == 0.0 and hi == 1.0


def test_choose_grouping():
    e = q.Env()
    e.column(abi.T_I32)
    e.column(abi.T_I64)
    aq = q.AggQuery(e, None, [(q.col(0), True)], [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True)])
    G = 1 << 22  # a global table of 4M slots (the engine keeps dense tables within 512 MB)
    rows = 1 << 20  # a quarter of the slots: the fewest rows the engine's rule takes a dense table for
    ds = E.choose_grouping(aq.plan, [(0, G - 1)], rows, None)  # no prediction: the engine's rule
    assert ds is not None and ds.G == G and not ds.priv and not ds.copies
    assert E.choose_grouping(aq.plan, [(0, G - 1)], rows, 5_000.0) is None and aq.plan.densePriv == 0
    ds = E.choose_grouping(aq.plan, [(0, G - 1)], rows, 400_000.0)  # groups a tenth of the slots: kept
    assert ds is not None and ds.G == G
    ds = E.choose_grouping(aq.plan, [(0, G - 1)], 10_000_000, 5_000.0)  # more rows than slots: kept
    assert ds is not None and ds.G == G
    ds = E.choose_grouping(aq.plan, [(0, 9)], 10_000_000, 3.0)  # private rows: never second-guessed
    assert ds is not None and ds.priv
