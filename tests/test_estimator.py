"""The group-count estimator on the CPU: the HyperLogLog definition against exact distinct counts, the
stored BF16 model against fresh synthetic tables (it must cut the naive sample scale-up's tail
errors), and the features' shape."""
import numpy as np

from warpstore_b200 import estimator as E
from warpstore_b200 import train_estimator as T


def test_hll_estimate_accuracy():
    rng = np.random.default_rng(0)
    for k in (10, 1_000, 100_000, 2_000_000):
        keys = rng.integers(0, 1 << 62, k).astype(np.uint64)
        est = E.hll_estimate(E.hll_registers(np.concatenate([keys, keys[: k // 2]])))
        assert abs(est - k) / k < 0.05, (k, est)


def test_model_beats_naive_scale_up():
    m = E.Model()
    rng = np.random.default_rng(123)  # tables the model has not seen (training seed 0)
    xs, ys = [], []
    for _ in range(24):
        x, y = T.make_example(rng, None, max_log2_rows=21)  # small tables: the CPU suite stays quick
        xs.append(x)
        ys.append(y)
    xs, ys = np.stack(xs), np.array(ys)
    pred = m.predict_log2_np(xs)
    err = np.abs(pred - ys)
    naive = np.abs(xs[:, 8] - ys)
    # sizing cares about the tail (an underestimated table overflows and reruns): the model must cut
    # the naive scale-up's large errors, and stay within ~1.2x at the median
    assert np.median(err) < 0.3
    assert np.quantile(err, 0.9) <= np.quantile(naive, 0.9) + 1e-6


def test_features_and_bf16_rounding():
    regs = E.hll_registers(np.arange(5000, dtype=np.uint64))
    x = E.features(regs, 10_000, 5_000, 1_000_000, 1e6)
    assert x.shape == (E.NFEATURES,) and np.all(np.isfinite(x))
    a = np.array([1.0, -2.5, 3.14159, 1e-8, 65504.0], dtype=np.float32)
    r = E.from_bf16(E.to_bf16(a))
    assert np.all(np.abs(r - a) <= np.abs(a) * 2 ** -8)
