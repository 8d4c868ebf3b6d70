"""Python mirror of the engine's GPU operator interface (src/gpu.h, src/jit.h) over the C ABI.

Names follow the reference: GpuAggregator (add_batch / run / run_window / overflowed / fetch / compact /
group_count), select / select_multi, gather_multi, hash_join / hash_join_parts, jit_get and the jit
modes.  Errors raise WsError with the engine's SQL error code.  Every call goes to libwarpstore_b200;
there is no host fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import WsError, check, lib

P = C.c_void_p


class DeviceBuffer:
    """A device allocation owned by Python (cudaMalloc through the library)."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = P()
        check(lib().ws_dev_alloc(max(self.nbytes, 1), C.byref(p)))
        self.ptr = p.value

    @classmethod
    def from_array(cls, a: np.ndarray) -> "DeviceBuffer":
        a = np.ascontiguousarray(a)
        b = cls(a.nbytes)
        if a.nbytes:
            check(lib().ws_h2d(b.ptr, a.ctypes.data, a.nbytes))
        return b

    def to_array(self, dtype, count: int | None = None) -> np.ndarray:
        dt = np.dtype(dtype)
        n = self.nbytes // dt.itemsize if count is None else count
        out = np.empty(n, dtype=dt)
        if n:
            check(lib().ws_d2h(out.ctypes.data, self.ptr, n * dt.itemsize))
        return out

    def free(self):
        if self.ptr:
            lib().ws_dev_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def device_to_array(ptr: int, dtype, count: int) -> np.ndarray:
    dt = np.dtype(dtype)
    out = np.empty(count, dtype=dt)
    if count:
        check(lib().ws_d2h(out.ctypes.data, ptr, count * dt.itemsize))
    return out


def tmp_free(ptr: int):
    if ptr:
        check(lib().ws_tmp_free(ptr))


def gpu_init():
    check(lib().ws_gpu_init())


def sync():
    check(lib().ws_gpu_sync())


TUNE_USE, TUNE_ON, TUNE_OFF = 0, 1, 2


def tune_set_mode(mode: int):
    """Launch-shape autotuner: TUNE_ON tunes unseen (kernel, plan, size class) keys inside ws_agg_run;
    TUNE_USE applies recorded choices; TUNE_OFF uses the default shapes."""
    check(lib().ws_tune_set_mode(int(mode)))


def tune_table() -> dict:
    """{key: (ctas per SM, shared KB, tile stages, join slots per key, microseconds)} of the autotuner's
    table (stages -1 and slots 0: the defaults)."""
    need = C.c_size_t()
    lib().ws_tune_table(None, 0, C.byref(need))
    buf = C.create_string_buffer(need.value)
    check(lib().ws_tune_table(buf, need.value, C.byref(need)))
    out = {}
    for line in buf.value.decode().splitlines():
        k, c, m, st, sl, us = line.split()
        out[k] = (int(c), int(m), int(st), int(sl), float(us))
    return out


def tune_clear():
    check(lib().ws_tune_clear())


def kernel_launches() -> int:
    return int(lib().ws_kernel_launches())


# ------------------------------------------------------------------ compiled plans
def jit_set_mode(mode: int):
    check(lib().ws_jit_set_mode(mode))


def jit_set_default_mode(mode: int):
    check(lib().ws_jit_set_default_mode(mode))


def jit_set_cache_dir(path: str):
    check(lib().ws_jit_set_cache_dir(path.encode()))


def jit_get(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, fn: int, kind: str = "") -> int | None:
    out = P()
    check(lib().ws_jit_get(C.byref(env), ncols, C.byref(plan), fn, kind.encode(), C.byref(out)))
    return out.value


def jit_info(prog: int) -> abi.JitInfo:
    info = abi.JitInfo()
    check(lib().ws_jit_program_info(prog, C.byref(info)))
    return info


def codegen_source(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, fn: int) -> str:
    need = C.c_size_t()
    check(lib().ws_codegen_source(C.byref(env), ncols, C.byref(plan), fn, None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib().ws_codegen_source(C.byref(env), ncols, C.byref(plan), fn, buf, need.value, C.byref(need)))
    return buf.value.decode()


def codegen_compile_check(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, fn: int, arch_sm: int = 100) -> int:
    n = C.c_size_t()
    check(lib().ws_codegen_compile_check(C.byref(env), ncols, C.byref(plan), fn, arch_sm, C.byref(n)))
    return n.value


# ------------------------------------------------------------------ aggregation
FETCH_STATUS = np.dtype([("groups", "<i8"), ("overflow", "<i4"), ("error", "<i4")])


class HostBuffer:
    """Pinned host memory that kernels can write (ws_host_alloc), viewed as a numpy array."""

    def __init__(self, shape, dtype):
        dtype = np.dtype(dtype)
        shape = tuple(int(x) for x in np.atleast_1d(shape))
        count = int(np.prod(shape))
        nbytes = max(count * dtype.itemsize, 1)
        p = P()
        check(lib().ws_host_alloc(nbytes, C.byref(p)))
        self.ptr = p.value
        raw = np.ctypeslib.as_array((C.c_uint8 * nbytes).from_address(self.ptr))
        self.array = raw[:count * dtype.itemsize].view(dtype).reshape(shape)

    def close(self):
        if self.ptr:
            self.array = None
            lib().ws_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Executor:
    """A prepared query (ws_exec_*): the aggregation of `plan` over device batches (the arrays of
    estimator.batch_arrays) built once with a CUDA graph of the whole query; run(env) queues it with
    env's constants, results() reads the groups after sync()."""

    def __init__(self, plan: abi.AggPlan, capacity: int, dense, env: abi.ExprEnv, ncols: int, arrays: tuple,
                 jit: int, max_groups: int):
        self.plan = plan
        self.h = None
        nb, bn, bdel, arr = arrays[:4]
        h = P()
        check(lib().ws_exec_create(C.byref(plan), int(capacity), C.byref(dense) if dense is not None else None,
                                   C.byref(env), ncols, nb, bn, bdel, arr, jit, int(max_groups), C.byref(h)))
        self.h = h.value
        self.max_groups = int(max_groups)

    def run(self, env: abi.ExprEnv):
        check(lib().ws_exec_run(self.h, C.byref(env)))

    def results(self):
        """(keys [g, nk] float64, exact [g, na, 2] int64, status) copies of the last run's groups."""
        k, x, s = P(), P(), P()
        check(lib().ws_exec_results(self.h, C.byref(k), C.byref(x), C.byref(s)))
        st = np.ctypeslib.as_array((C.c_uint8 * FETCH_STATUS.itemsize).from_address(s.value)).view(FETCH_STATUS)[0]
        g = min(int(st["groups"]), self.max_groups)
        nk, na = self.plan.nkeys, self.plan.naggs
        keys = np.ctypeslib.as_array((C.c_double * max(g * max(nk, 1), 1)).from_address(k.value))
        keys = keys[:g * nk].reshape(g, nk).copy()
        ex = np.ctypeslib.as_array((C.c_int64 * max(g * na * 2, 1)).from_address(x.value))[:g * na * 2]
        return keys, ex.reshape(g, na, 2).copy(), {n: int(st[n]) for n in FETCH_STATUS.names}

    def close(self):
        if self.h:
            lib().ws_exec_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ExecGroup:
    """Prepared queries of one compiled plan run as one graph with one multi-query scan
    (ws_exec_group_*): run(envs) queues them with one env each; each Executor's results() reads its
    groups after sync().  Close the group before its executors."""

    def __init__(self, executors: list, jit: int):
        self.executors = list(executors)
        self.h = None
        arr = (P * len(self.executors))(*[x.h for x in self.executors])
        h = P()
        check(lib().ws_exec_group_create(arr, len(self.executors), jit, C.byref(h)))
        self.h = h.value

    def run(self, envs: list):
        arr = (P * len(envs))(*[C.addressof(e) for e in envs])
        check(lib().ws_exec_group_run(self.h, arr))

    def close(self):
        if self.h:
            lib().ws_exec_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuAggregator:
    """GPU aggregation state of one query (src/gpu.h:84-130)."""

    def __init__(self, plan: abi.AggPlan, capacity: int, dense: abi.DenseSpec | None = None):
        self.plan = plan
        h = P()
        check(lib().ws_agg_create(C.byref(plan), int(capacity), C.byref(dense) if dense is not None else None,
                                  C.byref(h)))
        self.h = h.value

    def close(self):
        if self.h:
            lib().ws_agg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_batch(self, env: abi.ExprEnv, ncols: int, n: int, deleted: int = 0):
        check(lib().ws_agg_add_batch(self.h, C.byref(env), ncols, int(n), deleted or None))

    def add_batches(self, ncols: int, batches: list):
        """All batches at once: [(n, deleted_ptr, [ColView per column])]."""
        nb = len(batches)
        bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
        bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
        arr = _views_array([v for b in batches for v in b[2]])
        check(lib().ws_agg_add_batches(self.h, ncols, nb, bn, bdel, arr))

    def run(self, env: abi.ExprEnv, jit: int | None = None):
        check(lib().ws_agg_run(self.h, C.byref(env), jit))

    def run_window(self, env: abi.ExprEnv, jit: int | None = None):
        check(lib().ws_agg_run_window(self.h, C.byref(env), jit))

    def overflowed(self) -> bool:
        o = C.c_int()
        check(lib().ws_agg_overflowed(self.h, C.byref(o)))
        return bool(o.value)

    def group_count(self) -> int:
        g = C.c_int64()
        check(lib().ws_agg_group_count(self.h, C.byref(g)))
        return g.value

    def capacity(self) -> int:
        return int(lib().ws_agg_capacity(self.h))

    def batches(self) -> int:
        return int(lib().ws_agg_batches(self.h))

    def rows_in(self) -> int:
        return int(lib().ws_agg_rows_in(self.h))

    def is_dense(self) -> bool:
        return bool(lib().ws_agg_is_dense(self.h))

    def fetch(self, exact: bool = True):
        """(keys [g, nk] float64, accs [g, na] float64, exact [g, na, 2] int64 or None)."""
        nk, na = self.plan.nkeys, self.plan.naggs
        g = C.c_int64()
        rc = lib().ws_agg_fetch(self.h, 0, None, None, None, C.byref(g))
        if rc not in (0, 1206):
            check(rc)
        n = g.value
        keys = np.empty((n, nk), dtype=np.float64)
        accs = np.empty((n, na), dtype=np.float64)
        ex = np.empty((n, na, 2), dtype=np.int64) if exact else None
        check(lib().ws_agg_fetch(self.h, n, keys.ctypes.data if nk else None, accs.ctypes.data,
                                 ex.ctypes.data if exact else None, C.byref(g)))
        return keys, accs, ex

    def fetch_async(self, max_groups: int, keys: "HostBuffer | None", exact: "HostBuffer", status: "HostBuffer",
                    first: int = 0):
        """Queues the copy of groups [first, first + max_groups) straight into pinned host buffers
        (ws_agg_fetch_async); they are valid after sync().  status: a HostBuffer of FETCH_STATUS
        (all groups of the run, overflow, error)."""
        check(lib().ws_agg_fetch_async(self.h, int(first), int(max_groups), keys.ptr if keys is not None else None,
                                       exact.ptr, status.ptr))

    def sum_bits_slots(self) -> np.ndarray:
        out = np.zeros(self.plan.naggs, dtype=np.uint8)
        check(lib().ws_agg_sum_bits_slots(self.h, out.ctypes.data))
        return out

    def sum_high(self) -> np.ndarray:
        out = np.zeros(self.plan.naggs, dtype=np.int64)
        check(lib().ws_agg_sum_high(self.h, out.ctypes.data))
        return out

    def compact(self):
        """Groups left on the device, column-major: (keys_ptr, accs_ptr, g); free with tmp_free."""
        k, a, g = P(), P(), C.c_int64()
        check(lib().ws_agg_compact(self.h, C.byref(k), C.byref(a), C.byref(g)))
        return k.value, a.value, g.value


def agg_run_many(aggs: list, envs: list, jit: int | None = None):
    """One launch aggregating every aggregator over its batches (ws_agg_run_many)."""
    n = len(aggs)
    ha = (P * n)(*[a.h for a in aggs])
    he = (P * n)(*[C.addressof(e) for e in envs])
    check(lib().ws_agg_run_many(ha, he, jit, n))


def agg_nokeys_noalloc(env: abi.ExprEnv, ncols: int, plan: abi.AggPlan, batches: list, jit: int | None = None):
    """Filter + aggregate without GROUP BY through ws_agg_nokeys_noalloc (no memory is allocated: the
    library's fixed scratch array is used).  batches: [(n, deleted_ptr, [ColView])].  Returns the exact
    words [naggs, 2] (the layout of GpuAggregator.fetch's exact output)."""
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = [v for b in batches for v in b[2]]
    arr = _views_array(cols)
    out = np.zeros((plan.naggs, 2), dtype=np.int64)
    check(lib().ws_agg_nokeys_noalloc(C.byref(env), ncols, C.byref(plan), jit, nb, bn, bdel, arr, out.ctypes.data))
    return out


# ------------------------------------------------------------------ selection / gathers / joins
def _views_array(views: list) -> C.Array:
    arr = (abi.ColView * max(len(views), 1))()
    for i, v in enumerate(views):
        arr[i] = v
    return arr


def select_multi(env: abi.ExprEnv, where: abi.Prog | None, batches: list, ncols: int, jit: int | None = None):
    """batches: [(n, deleted_ptr, [ColView per column])].  Returns (idx_ptr, count, per_batch counts);
    idx_ptr holds ascending global indices into the concatenated batches (free with tmp_free)."""
    nb = len(batches)
    bn = (C.c_int64 * max(nb, 1))(*[b[0] for b in batches])
    bdel = (P * max(nb, 1))(*[b[1] or None for b in batches])
    cols = []
    for b in batches:
        cols.extend(b[2])
    arr = _views_array(cols)
    per = (C.c_int64 * max(nb, 1))()
    out = P()
    cnt = C.c_int64()
    check(lib().ws_select_multi(C.byref(env), 1 if where is not None else 0, where or abi.Prog(0, 0), nb, bn, bdel,
                                arr, ncols, C.byref(out), per, jit, C.byref(cnt)))
    return out.value, cnt.value, list(per)[:nb]


def gather_multi(views: list, boff: list, ptype: int, esize: int, idx_ptr: int, m: int, dst_ptr: int):
    arr = _views_array(views)
    bo = (C.c_int64 * max(len(boff), 1))(*boff)
    check(lib().ws_gather_multi(arr, bo, len(views), ptype, esize, idx_ptr, int(m), dst_ptr))


def gather(src_ptr: int, ptype: int, idx_ptr: int, m: int, dst_ptr: int):
    check(lib().ws_gather(src_ptr, ptype, idx_ptr, int(m), dst_ptr))


def hash_join_parts(build_key: abi.ColView, boff: list, probe_key: abi.ColView, poff: list):
    """Returns (build_idx_ptr, probe_idx_ptr, m, out_off); free the pointers with tmp_free."""
    bo = (C.c_int64 * len(boff))(*boff)
    po = (C.c_int64 * len(poff))(*poff)
    oo = (C.c_int64 * len(poff))()
    ob, op_ = P(), P()
    m = C.c_int64()
    check(lib().ws_hash_join_parts(build_key, bo, len(boff) - 1, probe_key, po, len(poff) - 1, C.byref(ob),
                                   C.byref(op_), oo, C.byref(m)))
    return ob.value, op_.value, m.value, list(oo)


def hash_join(build_key: abi.ColView, nb: int, probe_key: abi.ColView, np_: int):
    return hash_join_parts(build_key, [0, nb], probe_key, [0, np_])[:3]


def hash_join_sized(build_key: abi.ColView, nb: int, probe_key: abi.ColView, np_: int, first_capacity: int):
    """(build idx ptr, probe idx ptr, m, attempts) of the inner join whose pair buffers first hold
    first_capacity pairs (a second attempt with exact sizes when the join emits more)."""
    b, p, m, a = P(), P(), C.c_int64(), C.c_int()
    check(lib().ws_hash_join_sized(build_key, nb, probe_key, np_, int(first_capacity), C.byref(b), C.byref(p),
                                   C.byref(m), C.byref(a)))
    return b.value, p.value, m.value, a.value


def hash_join_outer(build_key: abi.ColView, nb: int, probe_key: abi.ColView, np_: int, full: bool = False):
    """(build idx ptr, probe idx ptr, m): unmatched probe rows pair with -1; `full` appends the build
    rows that matched nothing (probe -1).  Free the pointers with tmp_free."""
    b, p, m = P(), P(), C.c_int64()
    check(lib().ws_hash_join_outer(build_key, nb, probe_key, np_, int(full), C.byref(b), C.byref(p), C.byref(m)))
    return b.value, p.value, m.value


def cross_join(na: int, nb: int):
    a, b, m = P(), P(), C.c_int64()
    check(lib().ws_cross_join(na, nb, C.byref(a), C.byref(b), C.byref(m)))
    return a.value, b.value, m.value


def key_bitmap(key: abi.ColView, n: int, lo: int, nbits: int, bits_ptr: int):
    check(lib().ws_key_bitmap(key, n, lo, nbits, bits_ptr))


def set_bits(bits_ptr: int, idx_ptr: int, m: int):
    check(lib().ws_set_bits(bits_ptr, idx_ptr, m))


def remap_codes(in_ptr: int, n: int, map_ptr: int, map_n: int, out_ptr: int):
    check(lib().ws_remap_codes(in_ptr, n, map_ptr, map_n, out_ptr))


def bits_to_double(src_ptr: int, n: int, dst_ptr: int):
    check(lib().ws_bits_to_double(src_ptr, n, dst_ptr))


def gather_null(src_ptr: int, ptype: int, idx_ptr: int, m: int, dst_ptr: int):
    check(lib().ws_gather_null(src_ptr, ptype, idx_ptr, m, dst_ptr))


def gather_bytes(src_ptr: int, esize: int, idx_ptr: int, m: int, dst_ptr: int, nulls: bool = True):
    check(lib().ws_gather_bytes(src_ptr, esize, idx_ptr, m, dst_ptr, int(nulls)))


def gather_enc(view: abi.ColView, ptype: int, idx_ptr: int, m: int, dst_ptr: int):
    check(lib().ws_gather_enc(view, ptype, idx_ptr, m, dst_ptr))


def eval_at(env: abi.ExprEnv, ncols: int, prog: abi.Prog, idx_ptr: int | None, m: int, out_ptr: int):
    check(lib().ws_eval_at(C.byref(env), ncols, prog, idx_ptr, m, out_ptr))


def eval_at_int(env: abi.ExprEnv, ncols: int, prog: abi.Prog, idx_ptr: int | None, m: int, out_ptr: int):
    check(lib().ws_eval_at_int(C.byref(env), ncols, prog, idx_ptr, m, out_ptr))


def sort_perm(key_ptrs: list, desc: list, m: int) -> int:
    """Device pointer to the stable sort permutation (m int32) of rows by the double key columns
    (first = most significant); free with tmp_free."""
    kp = (P * max(len(key_ptrs), 1))(*key_ptrs)
    dp = (C.c_int * max(len(desc), 1))(*[int(d) for d in desc])
    out = P()
    check(lib().ws_sort_perm(kp, dp, len(key_ptrs), m, C.byref(out)))
    return out.value


def encode_column(src_ptr: int, t: int, n: int, enc: int = 0):
    """(device ptr, bytes, enc used) of an integer column encoded as one segment column (enc 7
    bit-packed, 8 run-length, 0 the smaller); free the pointer with tmp_free."""
    out, nb, used = P(), C.c_int64(), C.c_int()
    check(lib().ws_encode_column(src_ptr, t, n, enc, C.byref(out), C.byref(nb), C.byref(used)))
    return out.value, nb.value, used.value


def encode_column_engine(src_ptr: int, ptype: int, n: int):
    """(device ptr or None, bytes, enc) of a segment column in the engine's formats (enc 1-6, 0 = raw);
    free the pointer with tmp_free."""
    out, nb, used = P(), C.c_int64(), C.c_int()
    check(lib().ws_encode_column_engine(src_ptr, ptype, n, C.byref(out), C.byref(nb), C.byref(used)))
    return out.value, nb.value, used.value


def map_rank(keys_ptr: int, rank_ptr: int, m: int):
    check(lib().ws_map_rank(keys_ptr, rank_ptr, m))


# ---------------------------------------------------------------- tiered storage, UPDATE, distinct, temp columns
def set_vram_limit(nbytes: int):
    check(lib().ws_set_vram_limit(int(nbytes)))


def vram_used() -> int:
    return lib().ws_vram_used()


def place_column(host: np.ndarray, host_only: bool = False):
    """(device pointer, mapped) of a host column placed like the engine's placeColumn."""
    out, mapped = P(), C.c_int()
    check(lib().ws_place_column(host.ctypes.data, host.nbytes, int(host_only), C.byref(out), C.byref(mapped)))
    return out.value, bool(mapped.value)


def release_column(dev: int, host: np.ndarray, mapped: bool):
    check(lib().ws_release_column(dev, host.ctypes.data, host.nbytes, int(mapped)))


def vram_acquire(host: np.ndarray) -> int | None:
    out = P()
    check(lib().ws_vram_acquire(host.ctypes.data, host.nbytes, C.byref(out)))
    return out.value


def vram_release(dev: int, nbytes: int):
    check(lib().ws_vram_release(dev, nbytes))


def host_map(host: np.ndarray) -> int | None:
    out = P()
    check(lib().ws_host_map(host.ctypes.data, host.nbytes, C.byref(out)))
    return out.value


def host_unmap(host: np.ndarray):
    check(lib().ws_host_unmap(host.ctypes.data))


def patch_column(old_ptr: int, nbytes: int, width: int, rows: np.ndarray, vals: np.ndarray) -> int | None:
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    vals = np.ascontiguousarray(vals)
    out = P()
    check(lib().ws_patch_column(old_ptr, nbytes, width, rows.ctypes.data, vals.ctypes.data, rows.size, C.byref(out)))
    return out.value


def update_column(old_ptr: int, src_ptr: int, n: int, w: int, f64: bool, rows: np.ndarray, u: abi.Update) -> int | None:
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = P()
    check(lib().ws_update_column(old_ptr, src_ptr, n, w, int(f64), rows.ctypes.data, rows.size, C.byref(u), C.byref(out)))
    return out.value


def distinct_ints(env: abi.ExprEnv, ncols: int, prog: abi.Prog, idx_ptr: int | None, m: int, base: int,
                  span: int) -> np.ndarray:
    cap = max(1, min(span, m))
    out = np.empty(cap, dtype=np.int64)
    n = C.c_int64()
    check(lib().ws_distinct_ints(C.byref(env), ncols, prog, idx_ptr, m, base, span, out.ctypes.data, cap, C.byref(n)))
    return out[:n.value]


def bits_from_column(col_ptr: int, out: int, n: int, base: int, nbits: int):
    """(device pointer of the bitmap (ws_dev_free), saw_null)."""
    bits, nul = P(), C.c_int()
    check(lib().ws_bits_from_column(col_ptr, out, n, base, nbits, C.byref(bits), C.byref(nul)))
    return bits.value, bool(nul.value)


def temp_column(keys_ptr: int, nk: int, accs_ptr: int, na: int, g: int, spec: abi.TempColSpec):
    """(device pointer of the column (ws_dev_free), mn, mx)."""
    col, mn, mx = P(), C.c_double(), C.c_double()
    check(lib().ws_temp_column(keys_ptr, nk, accs_ptr, na, g, C.byref(spec), C.byref(col), C.byref(mn), C.byref(mx)))
    return col.value, mn.value, mx.value


def sort_perm_host(col: np.ndarray, ptype: int) -> np.ndarray:
    col = np.ascontiguousarray(col)
    perm = np.empty(max(col.size, 1), dtype=np.int32)
    check(lib().ws_sort_perm_host(col.ctypes.data, ptype, col.size, perm.ctypes.data))
    return perm[:col.size]


__all__ = ["DeviceBuffer", "Executor", "GpuAggregator", "WsError", "agg_nokeys_noalloc", "bits_to_double", "codegen_compile_check",
           "codegen_source", "cross_join", "device_to_array", "encode_column", "eval_at", "eval_at_int", "gather", "gather_bytes",
           "gather_enc", "gather_multi", "gather_null", "gpu_init", "hash_join", "hash_join_outer", "hash_join_parts",
           "jit_get", "jit_info", "jit_set_cache_dir", "jit_set_default_mode", "jit_set_mode", "kernel_launches",
           "key_bitmap", "map_rank", "remap_codes", "select_multi", "set_bits", "sort_perm", "sync", "tmp_free",
           "set_vram_limit", "vram_used", "place_column", "release_column", "vram_acquire", "vram_release", "host_map",
           "host_unmap", "patch_column", "update_column", "distinct_ints", "bits_from_column", "temp_column",
           "sort_perm_host", "encode_column_engine", "agg_run_many"]
