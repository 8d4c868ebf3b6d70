"""Learned cardinality estimator: group counts, filter selectivity and join output size.

Three predictions, each from a few statistics that one cheap GPU pass (or the segment metadata) gives
and a small MLP (F -> 64 -> 64 -> 1, BF16 weights, FP32 accumulation, run by `ws_mlp_infer`) that
corrects a plain statistical estimate in the log2 domain:

* ``groups`` -- the group count of a GROUP BY, to size its hash table: a HyperLogLog sketch (2^12
  registers) of a strided sample of the rows that pass the filter (`ws_hll_sketch`), the row counts
  and the keys' value range; the plain estimate extrapolates the sample's distinct count as if the
  values were equally frequent.
* ``rows`` -- the rows a filter passes, to size a selection's index buffer or a join's build side: the
  same sampled pass (without keys it only counts), plus zone maps -- each segment's min / max of the
  columns the filter compares with constants (``col < c``, ``col >= c``, ``col = c`` ...) bound and
  interpolate the fraction of rows that pass; the plain estimate is the sample's fraction scaled up.
* ``pairs`` -- the pairs an inner equi-join emits, to size its pair buffers: a coordinated sample of
  both sides (every row whose key hash falls below one threshold, ~2^16 rows of the larger side) whose
  join, scaled up, is the plain estimate; HyperLogLog sketches of the build and the probe keys (their
  registers' maximum sketches the union, so inclusion-exclusion gives the shared distinct keys) add
  probe rows x containment x build rows per distinct key, which stays informative where the sample
  holds few pairs.

Counts are compared in log2(1 + count) with a floor of 1024 (the smallest capacity any of them sizes).
The correction is applied only where the MLP moves the estimate by more than a gate chosen on
validation tables (``gate``): where the plain estimate is already right (a saturated sample, a filter
the zone maps decide), the plain estimate stands.  Sizing is never trusted for results: a table or a
buffer that turns out too small is regrown and the work repeated, so an estimate only changes how many
runs an operator takes and how much memory it holds.

The weights (`estimator_weights.npz`, prefixes "" / "rows_" / "pairs_") come from `train_estimator.py`:
synthetic tables with the exact counts as labels.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HLL_P = 12
NFEATURES = 10  # the group-count model's inputs
# Every capacity the estimates size starts at 1024 entries, so counts below that are the same to it:
# predictions, labels and errors are taken in log2(1 + max(count, 1024)).
FLOOR_LOG2 = math.log2(1 + 1024)
HIDDEN = 64
TARGETS = ("groups", "rows", "pairs")
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "estimator_weights.npz")


def prefix_of(target: str) -> str:
    if target not in TARGETS:
        raise ValueError(f"unknown estimator target {target!r}")
    return "" if target == "groups" else target + "_"


# ---------------------------------------------------------------- sketch (definition shared with the GPU)
def mix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer over uint64 (the hash of the GPU kernels)."""
    z = np.asarray(x).astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def sample_rows_of(total: int, sample_rows: int) -> np.ndarray:
    """Global rows the sketch samples: k * stride, stride = max(1, total // sample_rows)."""
    stride = max(1, total // max(sample_rows, 1)) if sample_rows > 0 else 1
    return np.arange(0, total, stride, dtype=np.int64)


def clz64(x: np.ndarray) -> np.ndarray:
    """Leading zero bits of uint64 values (64 for 0)."""
    x = x.astype(np.uint64)
    n = np.zeros(x.shape, dtype=np.int64)
    for s in (32, 16, 8, 4, 2, 1):
        top = (x >> np.uint64(64 - s)) == 0
        n += np.where(top, s, 0)
        x = np.where(top, x << np.uint64(s), x)
    return np.where(x == 0, 64, n)


def hll_registers(key_bits: np.ndarray, p: int = HLL_P) -> np.ndarray:
    """Registers of the keys' sketch: index = top p bits of mix64(key), value = leading zeros of the
    rest + 1 (the GPU kernel's definition, for a single integer key)."""
    h = mix64(key_bits.astype(np.uint64))
    j = (h >> np.uint64(64 - p)).astype(np.int64)
    rest = h << np.uint64(p)
    rank = np.where(rest == 0, 64 - p + 1, clz64(rest) + 1).astype(np.uint32)
    regs = np.zeros(1 << p, dtype=np.uint32)
    np.maximum.at(regs, j, rank)
    return regs


def hll_estimate(regs: np.ndarray) -> float:
    """Distinct-count estimate of a sketch (Flajolet et al. 2007, with linear counting for small
    cardinalities)."""
    m = regs.size
    alpha = 0.7213 / (1 + 1.079 / m)
    e = alpha * m * m / float(np.sum(np.ldexp(1.0, -regs.astype(np.int64))))
    zeros = int(np.sum(regs == 0))
    if e <= 2.5 * m and zeros:
        e = m * math.log(m / zeros)
    return e


# ---------------------------------------------------------------- features: group counts
def uniform_distinct(d: float, s: float) -> float:
    """The distinct values D of a population with equally frequent values whose sample of s rows shows d
    of them: the root of D (1 - exp(-s / D)) = d (increasing in D from 0 towards s), by bisection on
    log D.  Infinite (nothing bounds D) when d is within 5 % of s: the sketch's error (1.6 % at 2^12
    registers) cannot tell such a sample from one whose rows are all distinct."""
    if d <= 0:
        return 0.0
    if d >= 0.95 * s:
        return math.inf
    lo, hi = d, d * 2.0 ** 60
    for _ in range(100):
        mid = math.sqrt(lo * hi)
        if mid * -math.expm1(-s / mid) < d:
            lo = mid
        else:
            hi = mid
    return hi


def features(regs: np.ndarray, sampled: int, passing: int, total_rows: int, key_range: float | None) -> np.ndarray:
    """The group-count model's inputs (log2 domain where counts are concerned).  The last one is the
    plain estimate: the sample's distinct count d extrapolated as if the values were equally frequent
    (uniform_distinct; a saturated sample, whose d barely grows with more rows, stays near d), at most d
    scaled up by the sampling rate, the passing rows and the key range."""
    est = hll_estimate(regs)
    scale = total_rows / max(sampled, 1)
    kr = float(key_range) if key_range else 2.0 ** 63
    scaled = min(est * scale, passing * scale, kr)
    naive = min(uniform_distinct(est, passing), scaled)
    zeros = float(np.mean(regs == 0))
    return np.array([
        math.log2(1 + est), math.log2(1 + passing), math.log2(1 + sampled), math.log2(1 + total_rows),
        min(math.log2(1 + kr), 64.0), est / max(passing, 1), passing / max(sampled, 1), zeros,
        math.log2(1 + scaled), math.log2(1 + naive)], dtype=np.float32)


# ---------------------------------------------------------------- features: filter selectivity
def range_terms(where) -> tuple[list, int]:
    """(terms, opaque) of a filter expression (query.Expr): its AND-ed conjuncts of the form ``column op
    constant`` or ``constant op column`` (op one of < <= > >= =) as (column slot, op, value) with the
    column on the left, and the number of other conjuncts (which zone maps cannot bound)."""
    from . import abi
    if where is None:
        return [], 0
    flip = {abi.OP_LT: abi.OP_GT, abi.OP_LE: abi.OP_GE, abi.OP_GT: abi.OP_LT, abi.OP_GE: abi.OP_LE,
            abi.OP_EQ: abi.OP_EQ}
    terms, opaque, stack = [], 0, [where]
    while stack:
        e = stack.pop()
        if e.op == abi.OP_AND:
            stack.extend(e.kids)
            continue
        if e.op in flip and len(e.kids) == 2:
            a, b = e.kids
            if a.op == abi.OP_COL and b.op == abi.OP_CONST:
                terms.append((a.arg, e.op, float(b.value)))
                continue
            if b.op == abi.OP_COL and a.op == abi.OP_CONST:
                terms.append((b.arg, flip[e.op], float(a.value)))
                continue
        opaque += 1
    return terms, opaque


def _term_fraction(op: int, c: float, mn: float, mx: float) -> tuple[float, float, float]:
    """(all, est, any) for a segment whose column values lie in [mn, mx]: all = 1 if every value passes
    ``x op c``, any = 0 if none can, est = the passing fraction if the values were spread evenly."""
    from . import abi
    if mn > mx:  # no non-NULL value: nothing passes a comparison
        return 0.0, 0.0, 0.0
    w = mx - mn
    if op == abi.OP_EQ:
        if c < mn or c > mx:
            return 0.0, 0.0, 0.0
        if w == 0:
            return 1.0, 1.0, 1.0
        return 0.0, min(1.0, 1.0 / (w + 1.0)), 1.0
    if op in (abi.OP_LT, abi.OP_LE):
        strict = op == abi.OP_LT
        if (mx < c) or (not strict and mx <= c):
            return 1.0, 1.0, 1.0
        if (mn >= c) if strict else (mn > c):
            return 0.0, 0.0, 0.0
        return 0.0, (c - mn) / w if w else 0.5, 1.0
    strict = op == abi.OP_GT
    if (mn > c) or (not strict and mn >= c):
        return 1.0, 1.0, 1.0
    if (mx <= c) if strict else (mx < c):
        return 0.0, 0.0, 0.0
    return 0.0, (mx - c) / w if w else 0.5, 1.0


def zone_fractions(terms: list, opaque: int, seg_rows: list, seg_minmax: dict) -> tuple[float, float, float, float]:
    """(lo, est, hi, straddle) fractions of the rows, from each segment's min / max of the terms'
    columns (seg_minmax[slot] = [(min, max) per segment]; a column without statistics bounds nothing):
    lo = rows of segments where every term holds for every row and no opaque term exists, hi = rows of
    segments that no term excludes, est = the evenly-spread estimate (terms independent), straddle = rows
    of segments that neither every term admits entirely nor some term excludes."""
    total = float(sum(seg_rows)) or 1.0
    lo = est = hi = straddle = 0.0
    for s, n in enumerate(seg_rows):
        a_all, a_est, a_any = 1.0, 1.0, 1.0
        for slot, op, c in terms:
            mm = seg_minmax.get(slot)
            if mm is None:
                a_all = 0.0
                continue
            t_all, t_est, t_any = _term_fraction(op, c, float(mm[s][0]), float(mm[s][1]))
            a_all, a_est, a_any = a_all * t_all, a_est * t_est, a_any * t_any
        if opaque:
            a_all = 0.0
        lo += n * a_all
        est += n * a_est
        hi += n * a_any
        straddle += n * (1.0 if a_any and not a_all else 0.0)
    return lo / total, est / total, hi / total, straddle / total


def row_features(sampled: int, passing: int, total_rows: int, zones: tuple, opaque: int) -> np.ndarray:
    """The selectivity model's inputs; the last one is the plain estimate (the sample's passing
    fraction scaled up)."""
    lo, est, hi, straddle = zones
    s = passing / max(sampled, 1)
    naive = s * total_rows
    return np.array([
        s, est, lo, hi, straddle, float(min(opaque, 3)), math.log2(1 + sampled), math.log2(1 + passing),
        math.log2(1 + total_rows), math.log2(1 + est * total_rows), math.log2(1 + naive)], dtype=np.float32)


# ---------------------------------------------------------------- features: join output size
PAIR_SAMPLE_ROWS = 1 << 16  # rows of the larger side that the coordinated sample keeps


def sample_tau(build_rows: int, probe_rows: int, rows: int = PAIR_SAMPLE_ROWS) -> int:
    """The hash threshold of a coordinated sample that keeps about `rows` rows of the larger side."""
    big = max(build_rows, probe_rows, 1)
    return min((1 << 64) - 1, int(2.0 ** 64 * min(1.0, rows / big)))


def sampled_pairs(build_h: np.ndarray, probe_h: np.ndarray) -> int:
    """Pairs of the join of two coordinated samples (arrays of key hashes, one per row)."""
    if build_h.size == 0 or probe_h.size == 0:
        return 0
    keys, counts = np.unique(build_h.astype(np.uint64), return_counts=True)
    at = np.minimum(np.searchsorted(keys, probe_h.astype(np.uint64)), keys.size - 1)
    hit = keys[at] == probe_h
    return int(counts[at][hit].sum())


def pair_features(build_regs: np.ndarray, probe_regs: np.ndarray, build_rows: int, probe_rows: int,
                  sample_pairs: int, tau: int) -> np.ndarray:
    """The join-size model's inputs, from full sketches of the build and probe keys and a coordinated
    sample of both sides (every row whose key hash is below tau); the last one is the plain estimate,
    the sample join's pairs scaled by 2^64 / tau.  The sketches give probe rows x the share of distinct
    probe keys that the build holds (inclusion-exclusion over the union sketch) x build rows per
    distinct build key, an estimate that stays informative where the sample holds few pairs."""
    db, dp = hll_estimate(build_regs), hll_estimate(probe_regs)
    du = hll_estimate(np.maximum(build_regs, probe_regs))
    inter = min(max(db + dp - du, 0.0), db, dp)
    contain = inter / max(dp, 1.0)
    mult = build_rows / max(db, 1.0)
    formula = probe_rows * contain * mult
    scaled = sample_pairs * (2.0 ** 64 / max(tau, 1))
    return np.array([
        math.log2(1 + build_rows), math.log2(1 + probe_rows), math.log2(1 + db), math.log2(1 + dp),
        math.log2(1 + du), contain, math.log2(max(mult, 1.0)), db / max(du, 1.0), dp / max(du, 1.0),
        math.log2(1 + formula), math.log2(1 + sample_pairs), math.log2(1 + scaled)], dtype=np.float32)


# ---------------------------------------------------------------- model
def to_bf16(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bits (round to nearest even)."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) >> np.uint32(16)).astype(np.uint16)


def from_bf16(h: np.ndarray) -> np.ndarray:
    return (h.astype(np.uint32) << np.uint32(16)).view(np.float32)


class Model:
    """One target's MLP: predict_log2 = plain (the last feature) + the correction where it exceeds the gate."""

    def __init__(self, path=WEIGHTS, target: str = "groups"):
        d = np.load(path) if isinstance(path, str) else path  # a file, or a dict of its arrays
        files = list(d.keys())
        p = prefix_of(target)
        self.target = target
        self.w1, self.b1 = d[p + "w1"], d[p + "b1"].astype(np.float32)
        self.w2, self.b2 = d[p + "w2"], d[p + "b2"].astype(np.float32)
        self.w3, self.b3 = d[p + "w3"], float(d[p + "b3"])
        self.mean, self.std = d[p + "mean"].astype(np.float32), d[p + "std"].astype(np.float32)
        self.gate = float(d[p + "gate"]) if p + "gate" in files else 0.0
        self.meta = {k[len(p):]: d[k] for k in files if k.startswith(p + "val_")}
        self.nfeatures = int(self.mean.size)

    def normalise(self, x: np.ndarray) -> np.ndarray:
        return ((x - self.mean) / self.std).astype(np.float32)

    def forward_np(self, x: np.ndarray) -> np.ndarray:
        """Reference forward pass in FP32 over the BF16-rounded weights (tests, training checks)."""
        h = np.maximum(self.normalise(x) @ from_bf16(self.w1) + self.b1, 0)
        h = np.maximum(h @ from_bf16(self.w2) + self.b2, 0)
        return h @ from_bf16(self.w3) + np.float32(self.b3)

    def upper_log2(self, x: np.ndarray) -> np.ndarray:
        """What the count cannot exceed, from the features: a GROUP BY has at most as many groups as
        rows pass (the sample's passing fraction of the table) and as key values (the key range); a
        filter passes at most the table's rows."""
        x = x.astype(np.float64)
        if self.target == "groups":
            passing, sampled, total = np.exp2(x[:, 1]) - 1, np.exp2(x[:, 2]) - 1, np.exp2(x[:, 3]) - 1
            return np.minimum(np.log2(1 + passing * total / np.maximum(sampled, 1)), x[:, 4])
        if self.target == "rows":
            return x[:, 8]
        return np.full(x.shape[0], np.inf)

    def gated(self, x: np.ndarray, corr: np.ndarray) -> np.ndarray:
        corr = np.asarray(corr, dtype=np.float64)
        base = np.maximum(x[:, -1].astype(np.float64), FLOOR_LOG2)
        pred = np.minimum(base + np.where(np.abs(corr) > self.gate, corr, 0.0), self.upper_log2(x))
        return np.maximum(pred, FLOOR_LOG2)

    def predict_log2_np(self, x: np.ndarray) -> np.ndarray:
        """log2(1 + count), floored at 1024: the plain estimate (last feature) plus the gated MLP
        correction, at most upper_log2."""
        x = np.atleast_2d(x)
        return self.gated(x, self.forward_np(x))

    def predict_log2_gpu(self, x: np.ndarray) -> np.ndarray:
        x = np.atleast_2d(x)
        return self.gated(x, self.forward_gpu(x))

    def forward_gpu(self, x: np.ndarray) -> np.ndarray:
        from .ops import check, lib
        xn = np.ascontiguousarray(self.normalise(np.atleast_2d(x)))
        y = np.empty(xn.shape[0], dtype=np.float32)
        w1, w2, w3 = (np.ascontiguousarray(w) for w in (self.w1, self.w2, self.w3))
        check(lib().ws_mlp_infer(xn.ctypes.data, xn.shape[0], xn.shape[1], HIDDEN, w1.ctypes.data,
                                 self.b1.ctypes.data, w2.ctypes.data, self.b2.ctypes.data, w3.ctypes.data,
                                 C.c_float(self.b3), y.ctypes.data))
        return y

    def margin(self) -> float:
        """Capacity factor: 2^(90th percentile of the validation tables' underestimates in log2), the
        error that costs a rerun (an overestimate costs memory only)."""
        return 2.0 ** float(self.meta.get("p90_under_log2", self.meta.get("p90_log2_err", 0.0)))


_models: dict = {}


def model(target: str = "groups") -> Model:
    if target not in _models:
        _models[target] = Model(target=target)
    return _models[target]


# ---------------------------------------------------------------- on the device
def batch_arrays(batches: list):
    """The C arrays (nb, rows, deleted bitmaps, views) of device batches [(n, del_ptr, views)]."""
    from . import abi
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (C.c_void_p * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    return nb, bn, bdel, arr, sum(b[0] for b in batches)


def sketch(env, ncols: int, plan, batches, sample_rows: int = 1 << 18, p: int = HLL_P):
    """(registers, sampled rows, passing rows) of the GPU sketch over device batches (a list, or the
    arrays of batch_arrays).  A plan without GROUP BY keys only counts (registers all 0)."""
    from .ops import check, lib
    nb, bn, bdel, arr, _ = batches if isinstance(batches, tuple) else batch_arrays(batches)
    regs = np.zeros(1 << p, dtype=np.uint32)
    s, q = C.c_int64(), C.c_int64()
    check(lib().ws_hll_sketch(C.byref(env), ncols, C.byref(plan), nb, bn, bdel, arr, p, sample_rows,
                              regs.ctypes.data, C.byref(s), C.byref(q)))
    return regs, s.value, q.value


def estimate_groups(env, ncols: int, plan, batches: list, key_range: float | None = None,
                    sample_rows: int = 1 << 18) -> float:
    """Predicted group count of GROUP BY plan over the batches (GPU sketch + GPU MLP)."""
    regs, sampled, passing = sketch(env, ncols, plan, batches, sample_rows)
    total = batches[4] if isinstance(batches, tuple) else sum(b[0] for b in batches)
    x = features(regs, sampled, passing, total, key_range)
    return float(2.0 ** model().predict_log2_gpu(x)[0] - 1)


def estimate_rows(env, ncols: int, plan, where, batches: list, seg_minmax: dict | None = None,
                  sample_rows: int = 1 << 18) -> float:
    """Predicted rows that pass the filter of plan (built from the query.Expr `where`) over the batches:
    the GPU's sampled count, the zone maps of the batches (seg_minmax[slot] = [(min, max) per batch];
    None: no statistics) and the selectivity MLP on the GPU."""
    from . import abi
    counting = abi.AggPlan()
    C.memmove(C.addressof(counting), C.addressof(plan), C.sizeof(plan))
    counting.nkeys = 0
    _, sampled, passing = sketch(env, ncols, counting, batches, sample_rows)
    rows = [b[0] for b in batches] if not isinstance(batches, tuple) else list(batches[1][:batches[0]])
    terms, opaque = range_terms(where)
    x = row_features(sampled, passing, sum(rows), zone_fractions(terms, opaque, rows, seg_minmax or {}), opaque)
    return float(2.0 ** model("rows").predict_log2_gpu(x)[0] - 1)


def key_sketch(view, n: int, p: int = HLL_P) -> np.ndarray:
    """Sketch registers of every row of one key column (a device ColView of n rows)."""
    from . import abi
    from . import query as q
    e = q.Env()
    slot = e.column(view.t)
    aq = q.AggQuery(e, None, [(q.col(slot), True)], [q.Agg("COUNT")])
    regs, _, _ = sketch(e.env, e.ncols, aq.plan, [(n, 0, [view])], sample_rows=1 << 62, p=p)
    return regs


def key_sample(view, n: int, tau: int) -> np.ndarray:
    """The coordinated sample of one join key column (a device ColView of n rows): the hashes below tau."""
    from .ops import check, lib
    cap = max(1024, int(n * (tau / 2.0 ** 64) * 1.5) + 1024)
    while True:
        out = np.empty(cap, dtype=np.uint64)
        cnt = C.c_int64()
        check(lib().ws_join_key_sample(view, n, C.c_uint64(tau), out.ctypes.data, cap, C.byref(cnt)))
        if cnt.value <= cap:
            return out[:cnt.value]
        cap = cnt.value


def estimate_pairs(build_view, nb: int, probe_view, np_: int) -> float:
    """Predicted pairs of the inner equi-join of two key columns (device ColViews): sketches and a
    coordinated sample of both key columns on the GPU, the join-size MLP on the GPU."""
    tau = sample_tau(nb, np_)
    sp = sampled_pairs(key_sample(build_view, nb, tau), key_sample(probe_view, np_, tau))
    x = pair_features(key_sketch(build_view, nb), key_sketch(probe_view, np_), nb, np_, sp, tau)
    return float(2.0 ** model("pairs").predict_log2_gpu(x)[0] - 1)


def learned_capacity(pred_groups: float, min_cap: int = 1024) -> int:
    """Hash table capacity for a predicted group count: pow2 >= 2 x prediction x the model's margin,
    at least min_cap."""
    margin = model().margin()
    cap = min_cap
    while cap < 2 * pred_groups * margin:
        cap <<= 1
    return cap


def learned_pair_capacity(pred_pairs: float) -> int:
    """First pair-buffer capacity of a join for a predicted pair count (the prediction x the model's
    margin, rounded up to a multiple of 1024)."""
    c = int(math.ceil(pred_pairs * model("pairs").margin() * 1.05)) + 1024
    return (c + 1023) // 1024 * 1024


def choose_grouping(plan, ranges: list, rows: int, pred_groups: float | None):
    """DenseSpec or None (hash) for GROUP BY keys with value ranges [lo, hi]: the engine's rule
    (query.dense_spec, src/engine_select.cpp:1172-1229), except that a dense table in global memory
    whose slots outnumber both the rows (SPARSE_DENSE_ROWS times) and the predicted groups
    (SPARSE_DENSE_RATIO times) is left for the hash path, whose table the prediction sizes: there the
    dense table's clearing and compaction, which grow with its slots, outweigh the scan.  Measured on a
    B200 (1M rows, 4M-slot key range): 1,000 groups 0.252 ms hashed against 0.300 ms dense, 300,000
    groups 1.77 against 3.01 ms; with as many rows as slots or more the dense table was as fast or faster
    (16M rows, 1,000 groups: 0.648 dense against 0.860 ms hashed), so it stays.  Results are identical
    either way."""
    from . import query as q
    ds = q.dense_spec(plan, ranges, rows)
    if ds is None or pred_groups is None or ds.priv or ds.copies:
        return ds
    if (ds.G >= SPARSE_DENSE_RATIO * max(pred_groups, 1.0) and ds.G >= SPARSE_DENSE_ROWS * max(rows, 1)
            and ds.G >= SPARSE_DENSE_MIN_G):
        plan.densePriv = 0
        return None
    return ds


# A dense global-memory table of G slots is replaced by the hash path when G is at least this many
# times the predicted group count, at least SPARSE_DENSE_ROWS times the rows and SPARSE_DENSE_MIN_G.
SPARSE_DENSE_RATIO = 16
SPARSE_DENSE_ROWS = 4
SPARSE_DENSE_MIN_G = 1 << 20
