"""Trains the estimator's three models (estimator.py) on synthetic tables and writes estimator_weights.npz.

groups -- n rows (2^16 .. 2^24, log-uniform), keys uniform over K values, Zipf(s in [0.6, 1.6]) over K
  ranks (K log-uniform 1 .. 2^27), or (Zipf key, uniform second key) pairs, mixed to sparse int64 keys;
  a filter keeps 5-100 % of the rows; the sketch samples 2^16 .. 2^19 rows.  Label: log2(1 + exact group
  count of the filtered table).
rows -- n rows (2^16 .. 2^23) in segments of 2^15 .. 2^18 rows, 1-3 columns each sorted (time-like),
  sorted with local disorder, uniform or log-normal; a filter of 1-2 range terms whose constants are
  drawn for passing fractions from 10^-5 to 1 (and, for 30 % of the tables, one opaque term that the zone
  maps cannot see); 20 % of the columns come without segment statistics; the sample has 2^15 .. 2^19
  rows.  Label: log2(1 + rows that pass).
pairs -- build 2^10 .. 2^22 rows with unique keys or 1-8 rows per key, probe 2^12 .. 2^23 rows of which
  a uniform share 0-100 % (uniform or Zipf over the build keys) matches and the rest holds keys absent
  from the build; sketches of every key of both sides and their coordinated sample.  Label: log2(1 +
  the inner join's pairs).

Each model: F -> 64 -> 64 -> 1, ReLU, predicting the correction to its plain estimate (the last
feature), Adam on the squared log2 error, weights stored rounded to BF16.  Counts, labels and errors
are floored at 1024 (estimator.FLOOR_LOG2): every capacity sized from them starts there.  The tables
split 70 / 15 / 15 into training, the gate's choice (the correction applies where it exceeds the
gate: of "never", the corrections' quantiles and 0, the one that minimises median + 90th percentile
|log2 error|, a smaller gate only where it does strictly better) and the reported validation figures
(median / p90 |log2 error| of the model and of the plain estimate, and the 90th percentile of
underestimates, the capacity margin).

    python -m warpstore_b200.train_estimator [--tables 400] [--seed 0] [--only groups,rows,pairs]
    python -m warpstore_b200.train_estimator --evaluate 200      # the error table on fresh tables
"""
from __future__ import annotations

import argparse
import math
import os

import numpy as np

from . import abi
from . import estimator as E


def zipf_ranks(rng, n, k, s):
    w = np.arange(1, k + 1, dtype=np.float64) ** -s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), k - 1)


def make_example(rng, sample_rows: int | None = None, max_log2_rows: float = 24):
    """(features, label) of one synthetic GROUP BY; sample_rows None: drawn from 2^16 .. 2^19."""
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


def segment_minmax(v: np.ndarray, seg: int) -> list:
    n = v.size
    full = n // seg * seg
    out = []
    if full:
        r = v[:full].reshape(-1, seg)
        out = list(zip(r.min(1).tolist(), r.max(1).tolist()))
    if full < n:
        out.append((float(v[full:].min()), float(v[full:].max())))
    return out


def make_rows_example(rng, sample_rows: int | None = None, max_log2_rows: float = 23):
    """(features, label) of one synthetic filter."""
    n = int(2 ** rng.uniform(16, max_log2_rows))
    seg = 1 << int(rng.integers(15, 19))
    if sample_rows is None:
        sample_rows = int(2 ** rng.uniform(15, 19))
    cols = []
    for _ in range(int(rng.integers(1, 4))):
        span = int(2 ** rng.uniform(4, 40))
        kind = int(rng.integers(0, 4))
        if kind == 0:  # sorted: arrival times, dates
            v = np.sort(rng.integers(0, span, n))
        elif kind == 1:  # mostly sorted (late arrivals)
            w = max(1, int(span * rng.uniform(0.001, 0.05)))
            v = np.sort(rng.integers(0, span, n)) + rng.integers(-w, w + 1, n)
        elif kind == 2:
            v = rng.integers(0, span, n)
        else:
            v = (rng.lognormal(0.0, rng.uniform(0.5, 2.0), n) * (span / 10.0)).astype(np.int64)
        cols.append(v.astype(np.float64))
    ops = [abi.OP_LT, abi.OP_LE, abi.OP_GT, abi.OP_GE, abi.OP_EQ]
    terms, mask = [], np.ones(n, dtype=bool)
    for _ in range(int(rng.integers(1, 3))):
        c = int(rng.integers(0, len(cols)))
        v = cols[c]
        op = ops[int(rng.choice(5, p=[0.25, 0.2, 0.25, 0.2, 0.1]))]
        frac = 10 ** rng.uniform(-5, 0)
        const = float(v[int(rng.integers(0, n))]) if op == abi.OP_EQ else \
            float(np.quantile(v, frac if op in (abi.OP_LT, abi.OP_LE) else 1 - frac))
        terms.append((c, op, const))
        mask &= {abi.OP_LT: v < const, abi.OP_LE: v <= const, abi.OP_GT: v > const, abi.OP_GE: v >= const,
                 abi.OP_EQ: v == const}[op]
    opaque = 0
    if rng.random() < 0.3:  # a term the zone maps cannot bound (a hash of the row, as x % m < k)
        opaque = 1
        mask &= (E.mix64(np.arange(n, dtype=np.uint64) + np.uint64(rng.integers(1, 1 << 40))) % np.uint64(1000)) < \
            np.uint64(rng.integers(20, 1000))
    truth = int(mask.sum())
    rows = E.sample_rows_of(n, sample_rows)
    seg_rows = [min(seg, n - s * seg) for s in range((n + seg - 1) // seg)]
    mm = {c: segment_minmax(cols[c], seg) for c in range(len(cols)) if rng.random() >= 0.2}
    zones = E.zone_fractions(terms, opaque, seg_rows, mm)
    x = E.row_features(rows.size, int(mask[rows].sum()), n, zones, opaque)
    return x, math.log2(1 + truth)


def make_pairs_example(rng, max_log2_rows: float = 23):
    """(features, label, probe rows) of one synthetic inner equi-join."""
    nb = int(2 ** rng.uniform(10, max_log2_rows - 1))
    npr = int(2 ** rng.uniform(12, max_log2_rows))
    unique = rng.random() < 0.6
    if unique:
        db = nb
        bids = rng.permutation(nb)
    else:
        db = max(1, int(nb / 2 ** rng.uniform(0, 3)))
        bids = rng.integers(0, db, nb)
    f = rng.uniform(0, 1) if rng.random() < 0.7 else 1.0
    if rng.random() < 0.5:
        matched = rng.integers(0, db, npr)
    else:
        matched = zipf_ranks(rng, npr, min(db, 1 << 22), rng.uniform(0.6, 1.4))
    other = db + rng.integers(0, int(2 ** rng.uniform(0, 30)), npr)
    pids = np.where(rng.random(npr) < f, matched, other)
    counts = np.bincount(bids, minlength=db)
    hit = pids < db
    truth = int(counts[pids[hit]].sum())
    base = np.uint64(rng.integers(1, 1 << 40))
    bkeys, pkeys = E.mix64(bids.astype(np.uint64) + base), E.mix64(pids.astype(np.uint64) + base)
    breg, preg = E.hll_registers(bkeys), E.hll_registers(pkeys)
    tau = E.sample_tau(nb, npr)
    bh, ph = E.mix64(bkeys), E.mix64(pkeys)  # the sampler's hash of each key, as the GPU computes it
    sp = E.sampled_pairs(bh[bh < np.uint64(tau)], ph[ph < np.uint64(tau)])
    return E.pair_features(breg, preg, nb, npr, sp, tau), math.log2(1 + truth), npr


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


def errors(pred, ys):
    """median and 90th percentile of |log2 error| above the sizing floor (1024)."""
    e = np.abs(np.maximum(pred, E.FLOOR_LOG2) - np.maximum(ys, E.FLOOR_LOG2))
    return float(np.median(e)), float(np.quantile(e, 0.9))


def fit(target: str, xs: np.ndarray, ys: np.ndarray, epochs: int, seed: int, extra_plain=None) -> dict:
    """Weights, gate and validation figures of one target (keys prefixed as estimator.Model reads them)."""
    n = len(ys)
    ntr, ntu = int(n * 0.7), int(n * 0.15)
    tr, tu, va = slice(0, ntr), slice(ntr, ntr + ntu), slice(ntr + ntu, n)
    floor = E.FLOOR_LOG2
    p, mean, std = train(xs[tr], np.maximum(ys[tr], floor) - np.maximum(xs[tr, -1], floor), E.HIDDEN, epochs, seed)
    pre = E.prefix_of(target)
    out = {"w1": E.to_bf16(p["w1"]), "b1": p["b1"].astype(np.float32), "w2": E.to_bf16(p["w2"]),
           "b2": p["b2"].astype(np.float32), "w3": E.to_bf16(p["w3"]), "b3": np.float32(p["b3"][0]),
           "mean": mean.astype(np.float32), "std": std.astype(np.float32), "gate": np.float32(0.0)}
    mdl = E.Model({pre + k: v for k, v in out.items()}, target)
    xt = xs[tu].astype(np.float32)
    corr = mdl.forward_np(xt)
    best = None
    # from "never" down to "always": a smaller gate is taken only where it does strictly better
    cands = [1e9] + [float(v) for v in np.quantile(np.abs(corr), np.linspace(0.95, 0.1, 18))] + [0.0]
    for g in cands:
        mdl.gate = g
        med, p90 = errors(mdl.predict_log2_np(xt), ys[tu])
        if best is None or med + p90 < best[0] - 1e-9:
            best = (med + p90, g)
    mdl.gate = best[1]
    out["gate"] = np.float32(best[1])
    xv = xs[va].astype(np.float32)
    pred = mdl.predict_log2_np(xv)
    med, p90 = errors(pred, ys[va])
    pm, pp = errors(xs[va, -1], ys[va])
    under = np.maximum(np.maximum(ys[va], floor) - pred, 0)
    out.update({"val_median_log2_err": np.float32(med), "val_p90_log2_err": np.float32(p90),
                "val_naive_median_log2_err": np.float32(pm), "val_naive_p90_log2_err": np.float32(pp),
                "val_p90_under_log2": np.float32(np.quantile(under, 0.9)), "val_tables": np.int32(n - ntr - ntu)})
    line = (f"{target:6s} ({n - ntr - ntu} validation tables): |log2 error| median {med:.3f}, p90 {p90:.3f}; "
            f"plain estimate median {pm:.3f}, p90 {pp:.3f}; gate {best[1]:.3f}")
    if extra_plain is not None:  # the plain sizing rule, where it differs from the plain estimate
        rm, rp = errors(extra_plain[va], ys[va])
        out.update({"val_rule_median_log2_err": np.float32(rm), "val_rule_p90_log2_err": np.float32(rp)})
        line += f"; sizing rule median {rm:.3f}, p90 {rp:.3f}"
    print(line)
    return {pre + k: v for k, v in out.items()}


def evaluate(n: int, seed: int) -> str:
    """A markdown table of |log2 error| (median / 90th percentile, floored at 1024) on n fresh tables per
    target: the naive rule (groups: the sample's distinct count scaled up; rows: the sample's passing
    fraction scaled up; pairs: the probe rows, the join's plain first capacity), the plain estimate
    (the model's base) and the model."""
    rng = np.random.default_rng(seed)
    lines = ["| target | tables | naive rule | plain estimate | learned (gated) | gate |", "|---|---|---|---|---|---|"]
    for target in E.TARGETS:
        m = E.Model(target=target)
        if target == "groups":
            data = [make_example(rng) for _ in range(n)]
            naive = np.array([d[0][8] for d in data])
        elif target == "rows":
            data = [make_rows_example(rng) for _ in range(n)]
            naive = np.array([d[0][-1] for d in data])
        else:
            data = [make_pairs_example(rng) for _ in range(n)]
            naive = np.array([math.log2(1 + d[2]) for d in data])
        xs = np.stack([d[0] for d in data]).astype(np.float32)
        ys = np.array([d[1] for d in data])
        cells = [errors(v, ys) for v in (naive, xs[:, -1].astype(np.float64), m.predict_log2_np(xs))]
        lines.append(f"| {target} | {n} | " + " | ".join(f"{a:.3f} / {b:.3f}" for a, b in cells) + f" | {m.gate:.3g} |")
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tables", type=int, default=400)
    ap.add_argument("--evaluate", type=int, default=0, help="only print the error table on this many fresh tables")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--only", default="groups,rows,pairs", help="targets to retrain (others are kept)")
    ap.add_argument("--out", default=E.WEIGHTS)
    a = ap.parse_args()
    if a.evaluate:
        print(evaluate(a.evaluate, a.seed + 777))
        return
    keep = {}
    if os.path.exists(a.out):
        d = np.load(a.out)
        keep = {k: d[k] for k in d.files}
    out = {}
    for i, target in enumerate(E.TARGETS):
        pre = E.prefix_of(target)
        if target not in a.only.split(","):
            out.update({k: v for k, v in keep.items()
                        if k.startswith(pre) and (pre or not any(k.startswith(E.prefix_of(t)) for t in E.TARGETS[1:]))})
            continue
        rng = np.random.default_rng(a.seed + 1000 * i)
        extra = None
        if target == "groups":
            data = [make_example(rng) for _ in range(a.tables)]
        elif target == "rows":
            data = [make_rows_example(rng) for _ in range(a.tables)]
        else:
            data = [make_pairs_example(rng) for _ in range(a.tables)]
            extra = np.array([math.log2(1 + d[2]) for d in data])
        xs = np.stack([d[0] for d in data]).astype(np.float64)
        ys = np.array([d[1] for d in data])
        out.update(fit(target, xs, ys, a.epochs, a.seed, extra))
    np.savez(a.out, **out)


if __name__ == "__main__":
    main()
