"""Trains the group-count estimator (estimator.py) on synthetic tables and writes estimator_weights.npz.

Tables: n rows (2^16 .. 2^24, log-uniform), keys uniform over K values, Zipf(s in [0.6, 1.6]) over
K ranks (K log-uniform 1 .. 2^27), or (Zipf key, uniform second key) pairs, mixed to sparse int64
keys; a filter keeps 5-100 % of the rows; the sketch samples 2^16 .. 2^19 rows.
Features: the sketch of the filtered keys of the sampled rows (estimator.features, the GPU kernel's
definition); label: log2(1 + exact group count of the filtered table).  Model: 9 -> 64 -> 64 -> 1,
ReLU, predicting the correction to the naive sample scale-up (feature 8), Adam on the squared log2
error; the weights are stored rounded to BF16.

    python -m warpstore_b200.train_estimator [--tables 400] [--seed 0]
"""
from __future__ import annotations

import argparse
import math

import numpy as np

from . import estimator as E


def zipf_ranks(rng, n, k, s):
    w = np.arange(1, k + 1, dtype=np.float64) ** -s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), k - 1)


def make_example(rng, sample_rows: int | None = None, max_log2_rows: float = 24):
    """(features, label) of one synthetic table; sample_rows None: drawn from 2^16 .. 2^19."""
    n = int(2 ** rng.uniform(16, max_log2_rows))
    if sample_rows is None:
        sample_rows = int(2 ** rng.uniform(16, 19))
    k = max(1, int(2 ** rng.uniform(0, 27)))
    u = rng.random()
    if u < 0.4 and k > 1:
        ranks = zipf_ranks(rng, n, min(k, 1 << 22), rng.uniform(0.6, 1.6))
    elif u < 0.6:  # (Zipf key, uniform second key) pairs: mostly distinct combinations, as GROUP BY (k, x)
        ranks = zipf_ranks(rng, n, min(max(k, 2), 1 << 22), rng.uniform(0.6, 1.6)) * (1 << 30) + \
            rng.integers(0, int(2 ** rng.uniform(10, 24)), n)
        k = 0  # no range statistics for a key pair
    else:
        ranks = rng.integers(0, k, n)
    keys = E.mix64(ranks.astype(np.uint64) + np.uint64(rng.integers(1, 1 << 40)))
    sel = rng.uniform(0.05, 1.0)
    mask = rng.random(n) < sel
    truth = np.unique(keys[mask]).size
    rows = E.sample_rows_of(n, sample_rows)
    sm = mask[rows]
    regs = E.hll_registers(keys[rows][sm])
    key_range = float(k) if k and rng.random() < 0.5 else None  # range statistics known or not
    x = E.features(regs, rows.size, int(sm.sum()), n, key_range)
    return x, math.log2(1 + truth)


def train(xs, ys, hidden, epochs, seed, decay=1e-4):
    rng = np.random.default_rng(seed)
    mean, std = xs.mean(0), xs.std(0) + 1e-6
    xn = (xs - mean) / std
    f = xs.shape[1]
    p = {"w1": rng.normal(0, math.sqrt(2 / f), (f, hidden)), "b1": np.zeros(hidden),
         "w2": rng.normal(0, math.sqrt(2 / hidden), (hidden, hidden)), "b2": np.zeros(hidden),
         "w3": rng.normal(0, math.sqrt(1 / hidden), hidden), "b3": np.zeros(1)}
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(v) for k, v in p.items()}
    lr, b1c, b2c = 3e-3, 0.9, 0.999
    for t in range(1, epochs + 1):
        h1p = xn @ p["w1"] + p["b1"]
        h1 = np.maximum(h1p, 0)
        h2p = h1 @ p["w2"] + p["b2"]
        h2 = np.maximum(h2p, 0)
        y = h2 @ p["w3"] + p["b3"][0]
        d = 2 * (y - ys) / len(ys)
        g = {"w3": h2.T @ d, "b3": np.array([d.sum()])}
        dh2 = np.outer(d, p["w3"]) * (h2p > 0)
        g["w2"], g["b2"] = h1.T @ dh2, dh2.sum(0)
        dh1 = dh2 @ p["w2"].T * (h1p > 0)
        g["w1"], g["b1"] = xn.T @ dh1, dh1.sum(0)
        for k in p:
            m[k] = b1c * m[k] + (1 - b1c) * g[k]
            v[k] = b2c * v[k] + (1 - b2c) * g[k] ** 2
            p[k] -= lr * ((m[k] / (1 - b1c ** t)) / (np.sqrt(v[k] / (1 - b2c ** t)) + 1e-8) + decay * p[k])
    return p, mean, std


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tables", type=int, default=400)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--sample-rows", type=int, default=0, help="0: drawn per table from 2^16 .. 2^19")
    ap.add_argument("--out", default=E.WEIGHTS)
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    data = [make_example(rng, a.sample_rows or None) for _ in range(a.tables)]
    xs = np.stack([d[0] for d in data]).astype(np.float64)
    ys = np.array([d[1] for d in data])
    nval = max(1, a.tables // 5)
    # residual model: the MLP learns the correction to the naive sample scale-up (feature 8)
    p, mean, std = train(xs[nval:], ys[nval:] - xs[nval:, 8], E.HIDDEN, a.epochs, a.seed)
    out = {"w1": E.to_bf16(p["w1"]), "b1": p["b1"].astype(np.float32), "w2": E.to_bf16(p["w2"]),
           "b2": p["b2"].astype(np.float32), "w3": E.to_bf16(p["w3"]), "b3": np.float32(p["b3"][0]),
           "mean": mean.astype(np.float32), "std": std.astype(np.float32)}
    np.savez(a.out, **out)
    mdl = E.Model(a.out)
    pred = mdl.predict_log2_np(xs[:nval].astype(np.float32))
    err = np.abs(pred - ys[:nval])
    naive = np.abs(xs[:nval, 8] - ys[:nval])
    out["val_median_log2_err"] = np.float32(np.median(err))
    out["val_p90_log2_err"] = np.float32(np.quantile(err, 0.9))
    out["val_naive_median_log2_err"] = np.float32(np.median(naive))
    out["val_naive_p90_log2_err"] = np.float32(np.quantile(naive, 0.9))
    out["val_tables"] = np.int32(nval)
    np.savez(a.out, **out)
    print(f"validation ({nval} tables): |log2 error| median {np.median(err):.3f}, p90 {np.quantile(err, 0.9):.3f}; "
          f"naive scale-up median {np.median(naive):.3f}, p90 {np.quantile(naive, 0.9):.3f}")


if __name__ == "__main__":
    main()
