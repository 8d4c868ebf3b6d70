"""The rest of the engine's src/gpu.h surface: tiered column storage (VRAM budget, mapped host columns),
column-level UPDATE copies, distinct integers of an expression, bitmaps of a column, temp-table
columns built from compacted groups, and the sort permutation of a host column — each against the
oracle or an exact numpy restatement of the engine's rule (src/gpu.cu:82-155, :229-369, :890-1016,
:1375-1386)."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q

pytestmark = pytest.mark.gpu

NULL32, NULL64 = abi.NULL_I32, abi.NULL_I64


@pytest.fixture(autouse=True)
def _device():
    ops.gpu_init()
    ops.set_vram_limit(2**63 - 1)
    yield
    ops.set_vram_limit(2**63 - 1)


def test_place_column_copies_within_budget_and_maps_beyond_it():
    rng = np.random.default_rng(1)
    a = rng.integers(-10**12, 10**12, 1 << 20, dtype=np.int64)
    used0 = ops.vram_used()
    ops.set_vram_limit(used0 + a.nbytes)
    d, mapped = ops.place_column(a)
    assert not mapped and ops.vram_used() == used0 + a.nbytes
    assert np.array_equal(ops.device_to_array(d, np.int64, a.size), a)
    b = rng.integers(0, 100, 1 << 16, dtype=np.int64)
    d2, mapped2 = ops.place_column(b)  # over the budget: the host bytes are mapped
    assert mapped2 and ops.vram_used() == used0 + a.nbytes
    assert np.array_equal(ops.device_to_array(d2, np.int64, b.size), b)
    ops.release_column(d2, b, mapped2)
    d3, mapped3 = ops.place_column(b, host_only=True)
    assert mapped3 and np.array_equal(ops.device_to_array(d3, np.int64, b.size), b)
    ops.release_column(d3, b, mapped3)
    ops.release_column(d, a, mapped)
    assert ops.vram_used() == used0
    ops.set_vram_limit(used0 + 10)
    assert ops.vram_acquire(a) is None  # does not fit: no copy, no error
    ops.set_vram_limit(2**63 - 1)
    v = ops.vram_acquire(a)
    assert v and ops.vram_used() == used0 + a.nbytes
    ops.vram_release(v, a.nbytes)
    assert ops.vram_used() == used0
    h = ops.host_map(b)
    assert h and np.array_equal(ops.device_to_array(h, np.int64, b.size), b)
    ops.host_unmap(b)
    assert 0.0 <= ops.lib().ws_vram_fill() <= 1.0 and ops.lib().ws_vram_free() > 0


@pytest.mark.parametrize("width", [4, 8])
def test_patch_column(width):
    rng = np.random.default_rng(2)
    dt = np.int32 if width == 4 else np.int64
    col = rng.integers(-1000, 1000, 100_003).astype(dt)
    rows = rng.choice(col.size, 5000, replace=False).astype(np.int32)
    vals = rng.integers(-10**6, 10**6, rows.size).astype(dt)
    d = ops.DeviceBuffer.from_array(col)
    used0 = ops.vram_used()
    p = ops.patch_column(d.ptr, col.nbytes, width, rows, vals)
    assert p and ops.vram_used() == used0 + col.nbytes
    want = col.copy()
    want[rows] = vals
    assert np.array_equal(ops.device_to_array(p, dt, col.size), want)
    assert np.array_equal(d.to_array(dt), col)  # the old copy is untouched
    ops.vram_release(p, col.nbytes)
    assert ops.patch_column(d.ptr, col.nbytes, 2, rows, vals) is None  # width 4 or 8 only


def update_np(old, src, rows, u, f64):
    """The engine's column UPDATE rule (src/gpu.cu:302-330) restated."""
    new = old.copy()
    bad = saw = False
    vals = []
    for r in rows:
        if f64:
            v = u.d0
            if u.kind:
                v = src[r]
                if np.isnan(v):
                    bad |= bool(u.not_null)
                    saw = True
                else:
                    v = v + u.add_d
            new[r] = v
            if not np.isnan(v):
                vals.append(v)
            continue
        v = u.i0
        if u.kind:
            v = int(src[r])
            if v == u.nul:
                bad |= bool(u.not_null)
                saw = True
            elif u.kind == 2:
                v += u.add
                if not -2**63 <= v < 2**63:
                    bad = True
                    v = (v + 2**63) % 2**64 - 2**63
        if v != u.nul and (v < u.lo or v > u.hi):
            bad = True
        new[r] = v
        if v != u.nul:
            vals.append(float(v))
    mn = min(vals) if vals else np.inf
    mx = max(vals) if vals else -np.inf
    return new, bad, saw, mn, mx


@pytest.mark.parametrize("case", ["const_i64", "copy_i32", "add_i64", "add_i64_out_of_range", "add_f64",
                                  "null_not_allowed"])
def test_update_column(case):
    rng = np.random.default_rng(3)
    n = 50_001
    f64 = case == "add_f64"
    w = 4 if case == "copy_i32" else 8
    if f64:
        old = rng.random(n)
        src = rng.random(n)
        src[rng.choice(n, 100, replace=False)] = np.nan
        dt = np.float64
    else:
        dt = np.int32 if w == 4 else np.int64
        null = NULL32 if w == 4 else NULL64
        old = rng.integers(-1000, 1000, n).astype(dt)
        src = rng.integers(-1000, 1000, n).astype(dt)
        src[rng.choice(n, 100, replace=False)] = null
    rows = rng.choice(n, 3000, replace=False).astype(np.int32)
    u = abi.Update()
    u.nul = int(NULL32 if w == 4 else NULL64)
    u.lo, u.hi = -10**9, 10**9
    if case == "const_i64":
        u.kind, u.i0 = 0, 77
    elif case == "copy_i32":
        u.kind = 1
    elif case == "add_i64":
        u.kind, u.add = 2, 5
    elif case == "add_i64_out_of_range":
        u.kind, u.add, u.hi = 2, 5, 900
    elif case == "add_f64":
        u.kind, u.add_d = 2, 0.25
    else:
        u.kind, u.not_null = 1, 1
    dold, dsrc = ops.DeviceBuffer.from_array(old), ops.DeviceBuffer.from_array(src)
    used0 = ops.vram_used()
    p = ops.update_column(dold.ptr, dsrc.ptr, n, w, f64, rows, u)
    want, bad, saw, mn, mx = update_np(old, src, rows, u, f64)
    assert bool(u.bad) == bad and bool(u.saw_null) == saw
    if bad:
        assert p is None and ops.vram_used() == used0
        return
    assert u.mn == mn and u.mx == mx
    got = ops.device_to_array(p, dt, n)
    assert np.array_equal(got, want, equal_nan=f64)
    ops.vram_release(p, old.nbytes)


def test_distinct_ints_matches_the_oracles_values():
    rng = np.random.default_rng(4)
    n = 200_000
    a = rng.integers(-500, 500, n, dtype=np.int32)
    a[rng.choice(n, 1000, replace=False)] = NULL32
    b = rng.integers(0, 3, n, dtype=np.int64)
    e = q.Env()
    ca = e.column(abi.T_I32N)
    cb = e.column(abi.T_I64)
    prog = e.compile(q.col(ca) * 3 + q.col(cb))
    da, db = ops.DeviceBuffer.from_array(a), ops.DeviceBuffer.from_array(b)
    e.bind(ca, da.ptr)
    e.bind(cb, db.ptr)
    idx = np.sort(rng.choice(n, n // 3, replace=False)).astype(np.int32)
    di = ops.DeviceBuffer.from_array(idx)
    base, span = -1000, 1800
    got = ops.distinct_ints(e.env, e.ncols, prog, di.ptr, idx.size, base, span)
    cols = [abi.ColView(a.ctypes.data, abi.T_I32N, 0, 0, 0), abi.ColView(b.ctypes.data, abi.T_I64, 0, 0, 0)]
    vals, ovf = oracle.eval_at(e.env, cols, prog, idx, idx.size, as_int=True)
    assert not ovf
    vals = vals[vals != NULL64]
    want = np.unique(vals[(vals >= base) & (vals < base + span)])
    assert np.array_equal(got, want)
    # every row (idx null)
    got_all = ops.distinct_ints(e.env, e.ncols, prog, None, n, base, span)
    vals, _ = oracle.eval_at(e.env, cols, prog, None, n, as_int=True)
    vals = vals[vals != NULL64]
    assert np.array_equal(got_all, np.unique(vals[(vals >= base) & (vals < base + span)]))
    # a program the engine does not evaluate exactly (a division) yields no values
    assert ops.distinct_ints(e.env, e.ncols, e.compile(q.col(ca) / 2), None, n, base, span).size == 0


@pytest.mark.parametrize("out", [0, 1])
def test_bits_from_column(out):
    rng = np.random.default_rng(5)
    n = 300_001
    dt, null = (np.int32, NULL32) if out == 0 else (np.int64, NULL64)
    col = rng.integers(-100, 5000, n).astype(dt)
    col[rng.choice(n, 10, replace=False)] = null
    d = ops.DeviceBuffer.from_array(col)
    base, nbits = 7, 4000
    bp, saw = ops.bits_from_column(d.ptr, out, n, base, nbits)
    words = ops.device_to_array(bp, np.uint32, (nbits + 31) // 32)
    ops.lib().ws_dev_free(bp)
    v = col[col != null].astype(np.int64) - base
    v = np.unique(v[(v >= 0) & (v < nbits)])
    want = np.zeros((nbits + 31) // 32, dtype=np.uint32)
    np.bitwise_or.at(want, v >> 5, (np.uint32(1) << (v & 31).astype(np.uint32)))
    assert saw and np.array_equal(words, want)


def temp_np(keys, accs, g, s):
    """The engine's temp-column rule (src/gpu.cu:904-950) restated in Python."""
    bits = lambda x: int(np.float64(x).view(np.int64))
    out, ints = [], []
    for r in range(g):
        A = lambda j: accs[j * g + r]
        nul = s.src == 1 and s.cnt >= 0 and A(s.cnt) == 0
        is_int, iv, dv = False, 0, 0.0
        if s.src == 0:
            k = keys[s.idx * g + r]
            if s.key_int:
                iv, is_int = bits(k), True
                nul = iv in (NULL64, NULL32)
            else:
                dv, nul = k, np.isnan(k)
        elif not nul:
            if s.kind == 1:
                iv, is_int = bits(A(s.idx)), True
            elif s.kind == 2:
                iv = (bits(A(s.hi)) * 2**32 + bits(A(s.idx)) + 2**63) % 2**64 - 2**63
                is_int = True
            elif s.kind == 3:
                iv, is_int = int(A(s.idx)), True
            elif s.kind == 4:
                if s.sum_bits:
                    sm = (float(bits(A(s.hi))) * 4294967296.0 + float(bits(A(s.idx)))) if s.hi >= 0 else float(bits(A(s.idx)))
                else:
                    sm = A(s.idx)
                dv = np.float64(sm) / np.float64(s.div) / np.float64(A(s.cnt))
            else:
                dv = np.float64(A(s.idx)) / np.float64(s.div)
                nul = np.isnan(dv)
        if s.mul != 1 and not nul:
            dv = (float(iv) if is_int else dv) * s.mul
            is_int = False
        if s.out == 2:
            out.append(np.nan if nul else (float(iv) if is_int else dv))
            continue
        v = 0 if nul else (iv if is_int else int(np.round(dv)) if abs(dv - np.trunc(dv)) != 0.5 else int(np.trunc(dv) + np.sign(dv)))
        if not nul:
            ints.append(v)
        out.append((NULL64 if s.out == 1 else NULL32) if nul else v)
    mn = float(min(ints)) if ints and s.out != 2 else -np.inf
    mx = float(max(ints)) if ints and s.out != 2 else np.inf
    return np.array(out, dtype=np.float64 if s.out == 2 else np.int64 if s.out == 1 else np.int32), mn, mx


@pytest.mark.parametrize("spec", [
    dict(src=0, idx=1, key_int=1, out=1), dict(src=0, idx=0, key_int=0, out=2), dict(src=1, kind=1, idx=2, out=1),
    dict(src=1, kind=2, idx=3, hi=4, out=1, cnt=0), dict(src=1, kind=3, idx=0, out=0),
    dict(src=1, kind=4, idx=3, hi=4, cnt=0, sum_bits=1, out=2, div=100.0), dict(src=1, kind=4, idx=5, cnt=0, out=2),
    dict(src=1, kind=0, idx=5, out=1, div=10.0), dict(src=1, kind=0, idx=5, out=2, mul=0.5)])
def test_temp_column(spec):
    rng = np.random.default_rng(6)
    g, nk, na = 5000, 2, 6
    keys = np.empty(nk * g)
    keys[:g] = rng.random(g) * 100
    keys[:g][rng.choice(g, 50, replace=False)] = np.nan
    ik = rng.integers(-10**6, 10**6, g, dtype=np.int64)
    ik[rng.choice(g, 50, replace=False)] = NULL64
    keys[g:] = ik.view(np.float64)
    accs = np.empty(na * g)
    cnt = rng.integers(0, 5, g).astype(np.float64)
    accs[:g] = cnt
    accs[g:2 * g] = rng.integers(0, 100, g).astype(np.float64)
    accs[2 * g:3 * g] = rng.integers(-10**15, 10**15, g, dtype=np.int64).view(np.float64)
    lo = rng.integers(0, 2**32, g, dtype=np.int64)
    hi = rng.integers(-1000, 1000, g, dtype=np.int64)
    accs[3 * g:4 * g] = lo.view(np.float64)
    accs[4 * g:5 * g] = hi.view(np.float64)
    accs[5 * g:] = rng.random(g) * 1000 - 500
    s = abi.TempColSpec()
    s.hi, s.cnt, s.div, s.mul = -1, -1, 1.0, 1.0
    for k, v in spec.items():
        setattr(s, k, v)
    dk, da = ops.DeviceBuffer.from_array(keys), ops.DeviceBuffer.from_array(accs)
    col, mn, mx = ops.temp_column(dk.ptr, nk, da.ptr, na, g, s)
    want, wmn, wmx = temp_np(keys, accs, g, s)
    got = ops.device_to_array(col, want.dtype, g)
    ops.lib().ws_dev_free(col)
    if s.out == 2:  # DOUBLE results: within the stated 1e-12 relative tolerance (contraction may differ)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    else:
        assert np.array_equal(got, want)
    assert (mn, mx) == (wmn, wmx)


@pytest.mark.parametrize("ptype", [abi.PT_I32, abi.PT_I64, abi.PT_F64])
def test_sort_perm_host_matches_the_oracle(ptype):
    rng = np.random.default_rng(7)
    n = 123_457
    if ptype == abi.PT_I32:
        col = rng.integers(-50, 50, n, dtype=np.int32)
    elif ptype == abi.PT_I64:
        col = rng.integers(-2**40, 2**40, n, dtype=np.int64)
        col[::7] = col[::7] % 13  # ties
    else:
        col = np.round(rng.random(n) * 100, 1)
        col[rng.choice(n, 500, replace=False)] = np.nan
    got = ops.sort_perm_host(col, ptype)
    want = oracle.sort_perm([col.astype(np.float64)], [False])
    assert np.array_equal(got, want)
