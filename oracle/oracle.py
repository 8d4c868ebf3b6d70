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
