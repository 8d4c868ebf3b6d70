"""ctypes wrapper of oracle/_ref/libwsref.so: the reference's own GPU operators (Warpstore src/gpu.cu and
src/jit.cu built for sm_100a; by default each aggregation / selection runs the reference's compiled plan,
set_compiled(False) its interpreted kernels) — TEST INFRASTRUCTURE ONLY, called by tests/."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from warpstore_b200 import abi

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libwsref.so")
P = C.c_void_p
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        l = C.CDLL(LIB)
        l.wsref_error.restype = C.c_char_p
        l.wsref_aggregate.argtypes = [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), C.POINTER(abi.DenseSpec),
                                      C.c_int64, C.c_int, P, P, P, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                      C.POINTER(C.c_float)]
        l.wsref_take.argtypes = [P, P, P]
        l.wsref_aggregate_compact.argtypes = [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan),
                                              C.POINTER(abi.DenseSpec), C.c_int64, C.c_int, P, P, P,
                                              C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(P), C.POINTER(P),
                                              C.POINTER(C.c_float)]
        l.wsref_hash_join.argtypes = [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.c_int64,
                                      C.POINTER(C.c_int64), P, P, C.POINTER(C.c_float)]
        l.wsref_select_multi.argtypes = [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, C.c_int, P, P, P, C.c_int,
                                         C.c_int64, C.POINTER(C.c_int64), P, P]
        l.wsref_gather.argtypes = [P, C.c_int, P, C.c_int64, P, C.POINTER(C.c_float)]
        l.wsref_hash_join_dev.argtypes = [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.POINTER(C.c_int64),
                                          C.POINTER(P), C.POINTER(P), C.POINTER(C.c_float)]
        l.wsref_free.argtypes = [P]
        l.wsref_select_multi_dev.argtypes = [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, C.c_int, P, P, P, C.c_int,
                                             C.POINTER(C.c_int64), C.POINTER(P), C.POINTER(C.c_float)]
        l.wsref_set_compiled.argtypes = [C.c_int]
        if l.wsref_init():
            raise RuntimeError(l.wsref_error().decode())
        _lib = l
    return _lib


def set_compiled(on: bool):
    """Compiled plans (the engine's production path, default) or the interpreted kernels."""
    lib().wsref_set_compiled(1 if on else 0)


def last_compiled() -> bool:
    """The calling thread's last aggregation / selection ran a compiled plan."""
    return bool(lib().wsref_last_compiled())


def _check(rc):
    if rc:
        raise RuntimeError("reference: " + lib().wsref_error().decode())


def aggregate(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, batches: list, dense=None, cap: int = 1024):
    """Reference GpuAggregator over device batches [(n, del_ptr, views)]: (keys [g, nk], accs [g, na],
    sum_high [na], overflowed, milliseconds of run()); when overflowed, (None, None, group count, True, ms)."""
    l = lib()
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    g = C.c_int64()
    ovf = C.c_int()
    ms = C.c_float()
    dp = C.byref(dense) if dense is not None else None
    _check(l.wsref_aggregate(C.byref(env), ncols, C.byref(plan), dp, cap, nb, bn, bdel, arr, C.byref(g), C.byref(ovf),
                             C.byref(ms)))
    if ovf.value:  # overflowed: the third element is the group count seen
        return None, None, g.value, True, ms.value
    n = g.value
    keys = np.zeros((n, plan.nkeys), dtype=np.float64)
    accs = np.zeros((n, plan.naggs), dtype=np.float64)
    hi = np.zeros(plan.naggs, dtype=np.int64)
    _check(l.wsref_take(keys.ctypes.data, accs.ctypes.data, hi.ctypes.data))
    return keys, accs, hi, bool(ovf.value), ms.value


def aggregate_compact(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, batches: list, dense=None, cap: int = 1024):
    """Reference GpuAggregator leaving the groups on the device: (keys_ptr, accs_ptr, g, overflowed, ms);
    free the pointers with free()."""
    l = lib()
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    g, ovf, ms = C.c_int64(), C.c_int(), C.c_float()
    k, a = P(), P()
    dp = C.byref(dense) if dense is not None else None
    _check(l.wsref_aggregate_compact(C.byref(env), ncols, C.byref(plan), dp, cap, nb, bn, bdel, arr, C.byref(g),
                                     C.byref(ovf), C.byref(k), C.byref(a), C.byref(ms)))
    return k.value, a.value, g.value, bool(ovf.value), ms.value


def hash_join(bk: abi.ColView, nb: int, pk: abi.ColView, np_: int):
    l = lib()
    m = C.c_int64()
    ms = C.c_float()
    _check(l.wsref_hash_join(bk, nb, pk, np_, 0, C.byref(m), None, None, C.byref(ms)))
    ob = np.empty(max(m.value, 1), dtype=np.int32)
    op = np.empty(max(m.value, 1), dtype=np.int32)
    _check(l.wsref_hash_join(bk, nb, pk, np_, m.value, C.byref(m), ob.ctypes.data, op.ctypes.data, C.byref(ms)))
    return ob[:m.value], op[:m.value], ms.value


def select_multi(env: abi.ExprEnv, where: abi.Prog | None, batches: list, ncols: int):
    l = lib()
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    m = C.c_int64()
    per = np.zeros(max(nb, 1), dtype=np.int64)
    hw = 1 if where is not None else 0
    w = where or abi.Prog(0, 0)
    _check(l.wsref_select_multi(C.byref(env), hw, w, nb, bn, bdel, arr, ncols, 0, C.byref(m), None, per.ctypes.data))
    idx = np.empty(max(m.value, 1), dtype=np.int32)
    _check(l.wsref_select_multi(C.byref(env), hw, w, nb, bn, bdel, arr, ncols, m.value, C.byref(m), idx.ctypes.data,
                                per.ctypes.data))
    return idx[:m.value], per[:nb]


def gather(src: int, ptype: int, idx: int, m: int, dst: int) -> float:
    ms = C.c_float()
    _check(lib().wsref_gather(src, ptype, idx, m, dst, C.byref(ms)))
    return ms.value


def hash_join_dev(bk: abi.ColView, nb: int, pk: abi.ColView, np_: int):
    """(build idx ptr, probe idx ptr, m, ms); free the pointers with free()."""
    m = C.c_int64()
    ob, op = P(), P()
    ms = C.c_float()
    _check(lib().wsref_hash_join_dev(bk, nb, pk, np_, C.byref(m), C.byref(ob), C.byref(op), C.byref(ms)))
    return ob.value, op.value, m.value, ms.value


def select_multi_dev(env: abi.ExprEnv, where, batches: list, ncols: int):
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = (abi.ColView * max(len(cols), 1))(*cols)
    m = C.c_int64()
    idx = P()
    ms = C.c_float()
    _check(lib().wsref_select_multi_dev(C.byref(env), 1 if where is not None else 0, where or abi.Prog(0, 0), nb, bn,
                                        bdel, arr, ncols, C.byref(m), C.byref(idx), C.byref(ms)))
    return idx.value, m.value, ms.value


def free(p: int):
    if p:
        lib().wsref_free(p)
