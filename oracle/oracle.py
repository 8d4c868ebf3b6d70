"""ctypes wrapper of the CPU oracle (oracle/ws_oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Used by tests/ as the parity checker and by bench.py's CPU-baseline leg; the product library never
calls it.  All inputs are host (numpy) buffers referenced by the same ABI structs the GPU operators take.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from warpstore_b200 import abi

from . import build as _build

P = C.c_void_p
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.LIB if os.path.exists(_build.LIB) else _build.build()
        l = C.CDLL(path)
        l.ws_oracle_aggregate.argtypes = [C.POINTER(abi.ExprEnv), C.POINTER(abi.AggPlan), C.c_int, P, P, P, C.c_int,
                                          C.c_int, C.POINTER(P)]
        l.ws_oracle_aggregate_distinct.argtypes = [C.POINTER(abi.ExprEnv), C.POINTER(abi.AggPlan), abi.Prog, C.c_int,
                                                   C.c_int, P, P, P, C.c_int, C.c_int, C.POINTER(P)]
        l.ws_oracle_prog_is_int.argtypes = [C.POINTER(abi.ExprEnv), abi.Prog]
        l.ws_oracle_encode_column_engine.argtypes = [P, C.c_int, C.c_int64, P, C.c_int64, C.POINTER(C.c_int64)]
        l.ws_oracle_ngroups.restype = C.c_int64
        l.ws_oracle_ngroups.argtypes = [P]
        l.ws_oracle_nkeys.argtypes = [P]
        l.ws_oracle_naggs.argtypes = [P]
        l.ws_oracle_overflow.argtypes = [P]
        l.ws_oracle_keys.argtypes = [P, P]
        l.ws_oracle_words.argtypes = [P, P]
        l.ws_oracle_free.argtypes = [P]
        l.ws_oracle_select.restype = C.c_int64
        l.ws_oracle_select.argtypes = [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, C.c_int, P, P, P, C.c_int, C.c_int,
                                       P, P]
        l.ws_oracle_hash_join.restype = C.c_int64
        l.ws_oracle_hash_join.argtypes = [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.c_int, P, P]
        l.ws_oracle_gather_multi.argtypes = [P, P, C.c_int, C.c_int, C.c_int, P, C.c_int64, P]
        l.ws_oracle_hash_join_outer.restype = C.c_int64
        l.ws_oracle_hash_join_outer.argtypes = [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.c_int, P, P]
        l.ws_oracle_sort_perm.argtypes = [P, P, C.c_int, C.c_int64, P]
        l.ws_oracle_eval_at.argtypes = [C.POINTER(abi.ExprEnv), P, abi.Prog, P, C.c_int64, C.c_int, P,
                                        C.POINTER(C.c_int)]
        l.ws_oracle_eval.restype = C.c_double
        l.ws_oracle_eval.argtypes = [C.POINTER(abi.ExprEnv), P, abi.Prog, C.c_int64, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib = l
    return _lib


def prog_is_int(env: abi.ExprEnv, prog: abi.Prog) -> bool:
    """The oracle's static type of an expression (int64 or double)."""
    r = lib().ws_oracle_prog_is_int(C.byref(env), prog)
    if r < 0:
        raise ValueError("malformed expression")
    return bool(r)


def encode_column_engine(col: np.ndarray, ptype: int):
    """(enc, bytes) of the engine's encoding of one segment column (enc 0: kept raw, bytes empty)."""
    col = np.ascontiguousarray(col)
    nb = C.c_int64()
    e = lib().ws_oracle_encode_column_engine(col.ctypes.data, ptype, col.size, None, 0, C.byref(nb))
    out = np.zeros(max(nb.value, 1), dtype=np.uint8)
    if e:
        lib().ws_oracle_encode_column_engine(col.ctypes.data, ptype, col.size, out.ctypes.data, out.size, C.byref(nb))
    return e, out[:nb.value] if e else out[:0]


def _batches(batches: list):
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    return nb, bn, bdel, arr


def _result(h) -> tuple[np.ndarray, np.ndarray, int]:
    l = lib()
    g, nk, na = l.ws_oracle_ngroups(h), l.ws_oracle_nkeys(h), l.ws_oracle_naggs(h)
    keys = np.zeros((g, nk), dtype=np.int64)
    words = np.zeros((g, na, 2), dtype=np.int64)
    if g and nk:
        l.ws_oracle_keys(h, keys.ctypes.data)
    if g:
        l.ws_oracle_words(h, words.ctypes.data)
    ovf = l.ws_oracle_overflow(h)
    l.ws_oracle_free(h)
    return keys, words, ovf


def aggregate(env: abi.ExprEnv, plan: abi.AggPlan, batches: list, ncols: int, nthreads: int = 0):
    """batches: [(n, deleted_ptr, [ColView])] over HOST memory.  Returns (keys [g, nk] int64 sorted,
    words [g, na, 2] int64, overflow flag)."""
    nb, bn, bdel, arr = _batches(batches)
    h = P()
    rc = lib().ws_oracle_aggregate(C.byref(env), C.byref(plan), nb, bn, bdel, arr, ncols,
                                   nthreads or os.cpu_count() or 1, C.byref(h))
    if rc:
        raise RuntimeError("oracle aggregate failed")
    return _result(h)


def aggregate_distinct(env: abi.ExprEnv, plan: abi.AggPlan, distinct: abi.Prog, distinct_int: bool, batches: list,
                       ncols: int, nthreads: int = 0):
    nb, bn, bdel, arr = _batches(batches)
    h = P()
    rc = lib().ws_oracle_aggregate_distinct(C.byref(env), C.byref(plan), distinct, int(distinct_int), nb, bn, bdel,
                                            arr, ncols, nthreads or os.cpu_count() or 1, C.byref(h))
    if rc:
        raise RuntimeError("oracle aggregate failed")
    return _result(h)


def select(env: abi.ExprEnv, where: abi.Prog | None, batches: list, ncols: int, nthreads: int = 0):
    nb, bn, bdel, arr = _batches(batches)
    l = lib()
    nt = nthreads or os.cpu_count() or 1
    m = l.ws_oracle_select(C.byref(env), 1 if where is not None else 0, where or abi.Prog(0, 0), nb, bn, bdel, arr,
                           ncols, nt, None, None)
    idx = np.empty(max(m, 1), dtype=np.int32)
    per = np.zeros(max(nb, 1), dtype=np.int64)
    l.ws_oracle_select(C.byref(env), 1 if where is not None else 0, where or abi.Prog(0, 0), nb, bn, bdel, arr, ncols,
                       nt, idx.ctypes.data, per.ctypes.data)
    return idx[:m], per[:nb]


def hash_join(build_key: abi.ColView, nb: int, probe_key: abi.ColView, np_: int, nthreads: int = 0):
    l = lib()
    nt = nthreads or os.cpu_count() or 1
    m = l.ws_oracle_hash_join(build_key, nb, probe_key, np_, nt, None, None)
    ob = np.empty(max(m, 1), dtype=np.int32)
    op = np.empty(max(m, 1), dtype=np.int32)
    l.ws_oracle_hash_join(build_key, nb, probe_key, np_, nt, ob.ctypes.data, op.ctypes.data)
    return ob[:m], op[:m]


def gather_multi(views: list, boff: list, ptype: int, esize: int, idx: np.ndarray, out: np.ndarray):
    arr = (abi.ColView * max(len(views), 1))(*views)
    bo = (C.c_int64 * max(len(boff), 1))(*boff)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    lib().ws_oracle_gather_multi(arr, bo, len(views), ptype, esize, idx.ctypes.data, len(idx), out.ctypes.data)


def eval_row(env: abi.ExprEnv, cols, prog: abi.Prog, row: int):
    """(value as double, int value, is_int, overflow) of one expression at one row."""
    iv = C.c_int64()
    ii = C.c_int()
    ov = C.c_int()
    arr = (abi.ColView * len(cols))(*cols)
    d = lib().ws_oracle_eval(C.byref(env), arr, prog, row, C.byref(iv), C.byref(ii), C.byref(ov))
    return d, iv.value, bool(ii.value), bool(ov.value)


def hash_join_outer(build_key: abi.ColView, nb: int, probe_key: abi.ColView, np_: int, full: bool):
    l = lib()
    m = l.ws_oracle_hash_join_outer(build_key, nb, probe_key, np_, int(full), None, None)
    ob = np.empty(max(m, 1), dtype=np.int32)
    op = np.empty(max(m, 1), dtype=np.int32)
    l.ws_oracle_hash_join_outer(build_key, nb, probe_key, np_, int(full), ob.ctypes.data, op.ctypes.data)
    return ob[:m], op[:m]


def sort_perm(keys: list, desc: list) -> np.ndarray:
    """Stable sort permutation of host double columns (first = most significant)."""
    keys = [np.ascontiguousarray(k, dtype=np.float64) for k in keys]
    m = len(keys[0]) if keys else 0
    kp = (P * max(len(keys), 1))(*[k.ctypes.data for k in keys])
    dp = (C.c_int * max(len(desc), 1))(*[int(d) for d in desc])
    perm = np.empty(max(m, 1), dtype=np.int32)
    lib().ws_oracle_sort_perm(kp, dp, len(keys), m, perm.ctypes.data)
    return perm[:m]


def eval_at(env: abi.ExprEnv, cols: list, prog: abi.Prog, idx, m: int, as_int: bool = False):
    """(values [m] float64 or int64, overflow flag) of one expression at rows idx (or 0..m-1)."""
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    out = np.empty(max(m, 1), dtype=np.int64 if as_int else np.float64)
    ix = None
    if idx is not None:
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        ix = idx.ctypes.data
    ov = C.c_int()
    lib().ws_oracle_eval_at(C.byref(env), arr, prog, ix, m, int(as_int), out.ctypes.data, C.byref(ov))
    return out[:m], bool(ov.value)


def compare_groups(plan: abi.AggPlan, okeys: np.ndarray, owords: np.ndarray, keys, exact: np.ndarray, g: int):
    """None when a GPU result equals the oracle's groups, else what differs.  keys [g][nkeys] float64 and
    exact [g][naggs][2] int64 are ws_agg_fetch's formats (integer keys as int64 bits); okeys / owords
    come from aggregate().  Integer slots and COUNT compare exactly (int128 words); DOUBLE slots within
    1e-12 relative."""
    if g != okeys.shape[0]:
        return f"{g} groups, the oracle has {okeys.shape[0]}"
    nk, na = plan.nkeys, plan.naggs
    if nk:
        gk = np.ascontiguousarray(keys[:g, :nk]).view(np.int64)
        o1, o2 = np.lexsort(gk.T[::-1]), np.lexsort(okeys.T[::-1])
        if not np.array_equal(gk[o1], okeys[o2]):
            return "group keys differ"
    else:
        o1 = o2 = np.arange(g)
    for a in range(na):
        mine, want = exact[:g][o1][:, a], owords[o2][:, a]
        if plan.aggInt[a] or plan.ops[a] == abi.AGG_COUNT:
            if not np.array_equal(mine, want):
                return f"slot {a} differs (exact words)"
            continue
        x, y = np.ascontiguousarray(mine[:, 0]).view(np.float64), np.ascontiguousarray(want[:, 0]).view(np.float64)
        if plan.ops[a] == abi.AGG_SUM:
            if not np.allclose(x, y, rtol=1e-12, atol=1e-300, equal_nan=True):
                return f"slot {a} differs beyond 1e-12 relative"
        elif not np.array_equal(x, y, equal_nan=True):
            return f"slot {a} differs"
    return None


def groupby_count_sum_np(key: np.ndarray, payload: np.ndarray, cut: int, s: np.ndarray | None = None):
    """WHERE payload < cut GROUP BY key: COUNT(*), SUM(payload)[, COUNT(DISTINCT s)] restated in numpy
    (a sort instead of a hash table; exact int64 sums, which hold while every group's sum is below 2^63).
    Returns [keys, counts, sums(, distinct counts)] sorted by key.  At 100M rows this takes seconds
    where aggregate()'s per-thread hash maps take minutes."""
    m = payload < cut
    k, p = key[m], payload[m]
    order = np.argsort(k)
    ks = k[order]
    starts = np.flatnonzero(np.concatenate(([True], ks[1:] != ks[:-1]))) if ks.size else np.zeros(0, np.int64)
    cnt = np.diff(np.append(starts, ks.size)).astype(np.int64)
    sums = np.add.reduceat(p[order], starts) if ks.size else np.zeros(0, np.int64)
    cols = [ks[starts], cnt, sums]
    if s is not None:
        gid = np.repeat(np.arange(starts.size, dtype=np.int64), cnt)
        sv = s[m][order].astype(np.int64)
        assert sv.size == 0 or (sv.min() >= 0 and sv.max() < (1 << 23))
        pairs = np.sort((gid << 23) | sv)
        first = np.concatenate(([True], pairs[1:] != pairs[:-1])) if pairs.size else np.zeros(0, bool)
        cols.append(np.bincount(pairs[first] >> 23, minlength=starts.size).astype(np.int64))
    return cols
