"""Comparison helpers of the parity tests: GPU aggregation results against the CPU oracle."""
from __future__ import annotations

import numpy as np

from warpstore_b200 import abi

DOUBLE_RTOL = 1e-12  # DOUBLE SUM / AVG: relative tolerance (FP64 summation order differs)


def slot_kinds(plan: abi.AggPlan):
    """Per slot: 'count', 'isum', 'imin', 'imax', 'dsum', 'dmin', 'dmax' (derived high halves as their partner)."""
    out = []
    for a in range(plan.naggs):
        op, i = plan.ops[a], plan.aggInt[a]
        if op == abi.AGG_COUNT:
            out.append("count")
        elif op == abi.AGG_SUM:
            out.append("isum" if i else "dsum")
        elif op == abi.AGG_MIN:
            out.append("imin" if i else "dmin")
        else:
            out.append("imax" if i else "dmax")
    return out


def as_i128(w: np.ndarray) -> list[int]:
    return [int(np.uint64(lo)) + (int(hi) << 64) for lo, hi in w.reshape(-1, 2)]


def sort_groups(keys_bits: np.ndarray, words: np.ndarray):
    if keys_bits.shape[0] == 0 or keys_bits.shape[1] == 0:
        return keys_bits, words
    order = np.lexsort(keys_bits.T[::-1])
    return keys_bits[order], words[order]


def compare_exact(plan: abi.AggPlan, gpu_keys: np.ndarray, gpu_exact: np.ndarray, ora_keys: np.ndarray,
                  ora_words: np.ndarray, extra_count_slot: bool = False):
    """Bit-exact keys, COUNT / integer SUM / MIN / MAX; doubles within DOUBLE_RTOL."""
    gk = np.ascontiguousarray(gpu_keys).view(np.int64) if gpu_keys.size else gpu_keys.astype(np.int64)
    gk, gx = sort_groups(gk.reshape(gpu_keys.shape), gpu_exact)
    ok, ow = sort_groups(ora_keys, ora_words)
    assert gk.shape == ok.shape, f"group count differs: gpu {gk.shape[0]} oracle {ok.shape[0]}"
    assert np.array_equal(gk, ok), "group keys differ"
    kinds = slot_kinds(plan) + (["count"] if extra_count_slot else [])
    for a, kind in enumerate(kinds):
        g, o = gx[:, a, :], ow[:, a, :]
        if kind in ("dsum",):
            gd = g[:, 0].view(np.float64)
            od = o[:, 0].view(np.float64)
            np.testing.assert_allclose(gd, od, rtol=DOUBLE_RTOL, atol=1e-300, err_msg=f"slot {a} ({kind})")
        elif kind in ("dmin", "dmax"):
            gd = g[:, 0].view(np.float64)
            od = o[:, 0].view(np.float64)
            assert np.array_equal(gd, od) or np.allclose(gd, od, rtol=0, atol=0), f"slot {a} ({kind})"
        elif kind == "isum":
            assert np.array_equal(g, o), f"slot {a} ({kind}) int128 sums differ"
        else:
            assert np.array_equal(g[:, 0], o[:, 0]), f"slot {a} ({kind}) differs"


def engine_sum(plan: abi.AggPlan, accs_row: np.ndarray, slot: int, hi_slot: int, sum_high=None) -> int:
    """Exact integer SUM as the engine's finalize recombines it from the fetch format
    (src/engine_core.h:1972-1990)."""
    bits = accs_row.view(np.int64)
    if hi_slot >= 0 and plan.aggBits[hi_slot]:
        return int(bits[hi_slot]) * (1 << 32) + int(bits[slot])
    if sum_high is not None:
        return (int(sum_high[slot]) << 64) + int(np.uint64(bits[slot]))
    return int(round(float(accs_row[slot])))
