"""Learned group-count estimator for sizing GROUP BY hash tables.

A HyperLogLog sketch (2^12 registers) of a strided sample of the rows that pass the filter, taken on
the GPU by `ws_hll_sketch`, plus the table's row count and key range, give nine features; a small MLP
(9 -> 64 -> 64 -> 1, BF16 weights, FP32 accumulation, run by `ws_mlp_infer`) corrects the naive
scale-up of the sample's distinct count (log2 domain) to the predicted group count.  The engine's plain sizing rule stays the fallback: a table that overflows is resized and
the run repeated, so the estimate only changes how many runs a query takes, never its result.

The weights (`estimator_weights.npz`) come from `train_estimator.py`: runs over synthetic tables
(uniform and Zipf keys, 65K-16.8M rows, selectivities 5-100 %) with the true group counts as labels.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HLL_P = 12
NFEATURES = 9
HIDDEN = 64
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "estimator_weights.npz")


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


def features(regs: np.ndarray, sampled: int, passing: int, total_rows: int, key_range: float | None) -> np.ndarray:
    """The estimator's inputs (log2 domain where counts are concerned)."""
    est = hll_estimate(regs)
    scale = total_rows / max(sampled, 1)
    kr = float(key_range) if key_range else 2.0 ** 63
    naive = min(est * scale, passing * scale, kr)
    zeros = float(np.mean(regs == 0))
    return np.array([
        math.log2(1 + est), math.log2(1 + passing), math.log2(1 + sampled), math.log2(1 + total_rows),
        min(math.log2(1 + kr), 64.0), est / max(passing, 1), passing / max(sampled, 1), zeros,
        math.log2(1 + naive)], dtype=np.float32)


# ---------------------------------------------------------------- model
def to_bf16(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bits (round to nearest even)."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) >> np.uint32(16)).astype(np.uint16)


def from_bf16(h: np.ndarray) -> np.ndarray:
    return (h.astype(np.uint32) << np.uint32(16)).view(np.float32)


class Model:
    def __init__(self, path: str = WEIGHTS):
        d = np.load(path)
        self.w1, self.b1 = d["w1"], d["b1"].astype(np.float32)
        self.w2, self.b2 = d["w2"], d["b2"].astype(np.float32)
        self.w3, self.b3 = d["w3"], float(d["b3"])
        self.mean, self.std = d["mean"].astype(np.float32), d["std"].astype(np.float32)
        self.meta = {k: d[k] for k in d.files if k.startswith("val_")}

    def normalise(self, x: np.ndarray) -> np.ndarray:
        return ((x - self.mean) / self.std).astype(np.float32)

    def forward_np(self, x: np.ndarray) -> np.ndarray:
        """Reference forward pass in FP32 over the BF16-rounded weights (tests, training checks)."""
        h = np.maximum(self.normalise(x) @ from_bf16(self.w1) + self.b1, 0)
        h = np.maximum(h @ from_bf16(self.w2) + self.b2, 0)
        return h @ from_bf16(self.w3) + np.float32(self.b3)

    def predict_log2_np(self, x: np.ndarray) -> np.ndarray:
        """log2(1 + groups): the naive sample scale-up (feature 8) plus the MLP's correction."""
        x = np.atleast_2d(x)
        return x[:, 8] + self.forward_np(x)

    def predict_log2_gpu(self, x: np.ndarray) -> np.ndarray:
        x = np.atleast_2d(x)
        return x[:, 8] + self.forward_gpu(x)

    def forward_gpu(self, x: np.ndarray) -> np.ndarray:
        from .ops import check, lib
        xn = np.ascontiguousarray(self.normalise(np.atleast_2d(x)))
        y = np.empty(xn.shape[0], dtype=np.float32)
        w1, w2, w3 = (np.ascontiguousarray(w) for w in (self.w1, self.w2, self.w3))
        check(lib().ws_mlp_infer(xn.ctypes.data, xn.shape[0], xn.shape[1], HIDDEN, w1.ctypes.data,
                                 self.b1.ctypes.data, w2.ctypes.data, self.b2.ctypes.data, w3.ctypes.data,
                                 C.c_float(self.b3), y.ctypes.data))
        return y


_model = None


def model() -> Model:
    global _model
    if _model is None:
        _model = Model()
    return _model


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
    arrays of batch_arrays)."""
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


def learned_capacity(pred_groups: float, min_cap: int = 1024) -> int:
    """Hash table capacity for a predicted group count: pow2 >= 2 x prediction x the model's 90th
    percentile error on its validation tables (an underestimate costs a rerun, an overestimate only
    table memory), at least min_cap."""
    margin = 2.0 ** float(model().meta.get("val_p90_log2_err", 0.0))
    cap = min_cap
    while cap < 2 * pred_groups * margin:
        cap <<= 1
    return cap
