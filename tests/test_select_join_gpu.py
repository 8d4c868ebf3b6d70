"""Parity of selection (ascending row indices + per-batch counts), gathers and inner hash joins with
the CPU oracle: indices bit-exact and in order; join pairs compared as sorted multisets."""
import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_select(t, e, where, jit, deleted=None):
    t.to_device()
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        prog = None
        if jit:
            fp = abi.AggPlan()
            fp.hasWhere = 1 if where is not None else 0
            if where is not None:
                fp.where = where
            fp.naggs = 1
            fp.ops[0] = abi.AGG_COUNT
            prog = ops.jit_get(e.env, e.ncols, fp, abi.JF_FLAGM, "filter")
            assert prog
        ptr, m, per = ops.select_multi(e.env, where, t.batches(True, [d.ptr for d in deleted] if deleted else None),
                                       e.ncols, prog)
        idx = ops.device_to_array(ptr, np.int32, m)
        ops.tmp_free(ptr)
        return idx, per
    finally:
        ops.jit_set_mode(-1)


@pytest.mark.parametrize("n", [0, 1, 1000, 1025, 3 * (1 << 20) + 17])
def test_select_multi(n):
    rng = np.random.default_rng(n)
    t = W.Table(max(n, 0))
    t.add("a", abi.T_I32, rng.integers(0, 2406, n, dtype=np.int32))
    t.add("b", abi.T_F64, rng.random(n))
    e = W.env_for(t)
    where = e.compile(q.and_(q.col(0).lt(1203), q.col(1).lt(q.lit(0.9))))
    if n == 0:
        ptr, m, per = ops.select_multi(e.env, where, [], e.ncols)
        assert m == 0
        ops.tmp_free(ptr)
        return
    oi, op = oracle.select(e.env, where, t.batches(False), e.ncols)
    for jit in (True, False):
        gi, gp = run_select(t, e, where, jit)
        assert np.array_equal(gi, oi)
        assert list(gp) == list(op)


def test_select_with_deletes_and_gather():
    n = 2 * (1 << 20) + 999
    rng = np.random.default_rng(1)
    t = W.Table(n)
    t.add("a", abi.T_I32, rng.integers(0, 100, n, dtype=np.int32))
    t.add("v", abi.T_I64, rng.integers(-2**40, 2**40, n, dtype=np.int64), enc=0)
    t.add("c", abi.T_I64, rng.integers(1000, 1200, n, dtype=np.int64), enc=1)
    e = W.env_for(t)
    where = e.compile(q.col(0).ge(50))
    dh, dd = [], []
    for s in range(t.nseg):
        m = t.seg_len(s)
        bits = rng.integers(0, 2**32, (m + 31) // 32, dtype=np.uint32) & rng.integers(0, 2**32, (m + 31) // 32, dtype=np.uint32)
        dh.append(bits)
        dd.append(ops.DeviceBuffer.from_array(bits))
    oi, op = oracle.select(e.env, where, t.batches(False, [d.ctypes.data for d in dh]), e.ncols)
    gi, gp = run_select(t, e, where, True, dd)
    assert np.array_equal(gi, oi) and list(gp) == list(op)
    # gathers of the selected rows: raw and encoded columns
    boff = [s * t.seg_rows for s in range(t.nseg)]
    idx = ops.DeviceBuffer.from_array(gi)
    for c, pt, es in ((1, abi.PT_I64, 8), (2, abi.PT_I64, 8), (0, abi.PT_I32, 4)):
        views = [t.views(s, True)[c] for s in range(t.nseg)]
        out = ops.DeviceBuffer(len(gi) * es)
        ops.gather_multi(views, boff, pt, es, idx.ptr, len(gi), out.ptr)
        got = out.to_array(np.int64 if es == 8 else np.int32)
        hv = [t.views(s, False)[c] for s in range(t.nseg)]
        want = np.empty(len(gi), dtype=got.dtype)
        oracle.gather_multi(hv, boff, pt, es, gi, want)
        assert np.array_equal(got, want)
        assert np.array_equal(got, t.cols[c].data[gi].astype(got.dtype))


def join_case(nb, np_, key_space, seed, dup=False, nulls=False, i32=False, sparse=False, shift=0):
    """Build / probe keys over [shift, shift + key_space); `sparse` spreads them over the whole integer
    range with an odd multiplier (a bijection), so the join takes the hash path, not the dense one."""
    rng = np.random.default_rng(seed)
    if dup:
        bk = rng.integers(0, key_space, nb)
    else:
        bk = rng.permutation(key_space)[:nb]
    pk = rng.integers(0, key_space, np_)
    bk, pk = bk.astype(np.int64) + shift, pk.astype(np.int64) + shift
    if sparse:
        mul = np.uint64(0x9E3779B97F4A7C15)
        bk, pk = (bk.astype(np.uint64) * mul).view(np.int64), (pk.astype(np.uint64) * mul).view(np.int64)
    dt = np.int32 if i32 else np.int64
    bk, pk = bk.astype(dt), pk.astype(dt)  # int32: keeps the low 32 bits (still a bijection of the keys)
    null = abi.NULL_I32 if i32 else abi.NULL_I64
    bk[bk == null] += 1
    pk[pk == null] += 1
    if nulls:
        bk[rng.random(nb) < 0.05] = null
        pk[rng.random(np_) < 0.05] = null
    return bk, pk


def check_join(bk, pk, i32):
    t = abi.T_I32N if i32 else abi.T_I64N
    nb, np_ = len(bk), len(pk)
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    ob, op, m = ops.hash_join(abi.ColView(db.ptr, t, 0, 0, 0), nb, abi.ColView(dp.ptr, t, 0, 0, 0), np_)
    gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
    ops.tmp_free(ob)
    ops.tmp_free(op)
    wb, wp = oracle.hash_join(abi.ColView(bk.ctypes.data, t, 0, 0, 0), nb, abi.ColView(pk.ctypes.data, t, 0, 0, 0), np_)
    assert m == len(wb)
    g = np.lexsort((gb, gp))
    w = np.lexsort((wb, wp))
    assert np.array_equal(gp[g], wp[w]) and np.array_equal(gb[g], wb[w])
    return m


@pytest.mark.parametrize("sparse", [False, True], ids=["dense-range", "hash"])
@pytest.mark.parametrize("nb,np_,space,dup,nulls,i32,shift", [
    (1000, 5000, 1000, False, False, False, 0),
    (100_000, 1_000_000, 400_000, False, False, False, 0),
    (50_000, 200_000, 10_000, True, True, False, 0),          # duplicate build keys: many matches per probe
    (30_000, 100_000, 30_000, False, True, True, 0),          # int32 keys with NULLs
    (40_000, 100_000, 60_000, True, False, False, -(1 << 40)),  # negative keys, duplicates
    (1, 1, 1, False, False, False, 0),
])
def test_hash_join(nb, np_, space, dup, nulls, i32, shift, sparse):
    bk, pk = join_case(nb, np_, space, nb + np_, dup, nulls, i32, sparse, shift)
    check_join(bk, pk, i32)


def test_hash_join_all_null_build_and_full_int64_range():
    pk = np.arange(-5, 5, dtype=np.int64)
    assert check_join(np.full(100, abi.NULL_I64, dtype=np.int64), pk, False) == 0
    bk = np.array([np.iinfo(np.int64).min + 1, np.iinfo(np.int64).max, 0, 3], dtype=np.int64)  # range = all of int64
    pk = np.array([3, np.iinfo(np.int64).max, 7, np.iinfo(np.int64).min + 1, 3], dtype=np.int64)
    assert check_join(bk, pk, False) == 4


def test_hash_join_multipass_matches_single_pass():
    """A table budget far below the build side forces the hash join into many passes (each pass builds
    the table of the build keys whose hash falls in it and probes every row); run in a child process
    because the budget is read once per process."""
    import subprocess
    import sys
    import os
    code = (
        "import numpy as np\n"
        "from tests.test_select_join_gpu import join_case, check_join\n"
        "bk, pk = join_case(100_000, 400_000, 300_000, 11, dup=True, nulls=True, sparse=True)\n"
        "print(check_join(bk, pk, False))\n")
    env = dict(os.environ, WARPSTORE_B200_JOIN_TABLE_BYTES=str(1 << 16))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert int(r.stdout.strip().splitlines()[-1]) > 0


FILTER_CASES = r"""
from tests.test_select_join_gpu import join_case, check_join
out = []
for nb, np_, space, dup, nulls, i32 in [(1000, 5000, 1000, False, False, False),
                                       (100_000, 1_000_000, 400_000, False, False, False),
                                       (50_000, 200_000, 10_000, True, True, False),
                                       (30_000, 100_000, 30_000, False, True, True), (1, 1, 1, False, False, False),
                                       (200_000, 600_000, 200_000, False, False, False)]:
    bk, pk = join_case(nb, np_, space, nb + np_, dup, nulls, i32, True)
    out.append(check_join(bk, pk, i32))
print(" ".join(map(str, out)))
"""


def test_hash_join_key_filter_matches_oracle():
    """The inner hash join's key filter (a blocked Bloom filter of the build keys that lets probes with
    no match skip their bucket), forced on for every size: the sparse-key cases above (duplicates, NULLs,
    int32 keys, every probe key matching) give the oracle's pairs.  A child process: the switch is read
    once per process."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, WARPSTORE_B200_JOIN_FILTER="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", FILTER_CASES], env=env, cwd=root, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    counts = [int(x) for x in r.stdout.strip().splitlines()[-1].split()]
    assert len(counts) == 6 and all(c > 0 for c in counts)


def test_sized_selective_join_uses_key_filter_same_pairs():
    """A first pair capacity well below the probe rows (a selective join: ~10 % of 3M probe rows match
    1.2M sparse build keys) turns the key filter on; the pairs equal the unfiltered join's."""
    rng = np.random.default_rng(17)
    mul = np.uint64(0x9E3779B97F4A7C15)
    bk = (rng.permutation(12_000_000)[:1_200_000].astype(np.uint64) * mul).view(np.int64)
    pk = (rng.integers(0, 12_000_000, 3_000_000).astype(np.uint64) * mul).view(np.int64)
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    bv, pv = abi.ColView(db.ptr, abi.T_I64, 0, 0, 0), abi.ColView(dp.ptr, abi.T_I64, 0, 0, 0)

    def pairs(ob, op, m):
        gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
        ops.tmp_free(ob)
        ops.tmp_free(op)
        o = np.lexsort((gb, gp))
        return gb[o], gp[o]

    want = pairs(*ops.hash_join(bv, len(bk), pv, len(pk)))
    ob, op, m, att = ops.hash_join_sized(bv, len(bk), pv, len(pk), 400_000)
    got = pairs(ob, op, m)
    assert att == 1 and m == want[0].size == int(np.isin(pk, bk).sum())
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_hash_join_partitions():
    rng = np.random.default_rng(4)
    P = 4
    bks, pks = [], []
    for p in range(P):  # co-located: partition p's keys are == p mod P
        b = (rng.permutation(20_000)[:5_000] * P + p).astype(np.int64)
        q = (rng.integers(0, 20_000, 30_000) * P + p).astype(np.int64)
        if p % 2:  # odd partitions sparse (hash path), even ones dense
            b, q = b * 0x3FFFFFFFFFF, q * 0x3FFFFFFFFFF
        bks.append(b)
        pks.append(q)
    bk, pk = np.concatenate(bks), np.concatenate(pks)
    boff = [0] + list(np.cumsum([len(x) for x in bks]))
    poff = [0] + list(np.cumsum([len(x) for x in pks]))
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    ob, op, m, outoff = ops.hash_join_parts(abi.ColView(db.ptr, abi.T_I64, 0, 0, 0), [int(x) for x in boff],
                                            abi.ColView(dp.ptr, abi.T_I64, 0, 0, 0), [int(x) for x in poff])
    gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
    ops.tmp_free(ob)
    ops.tmp_free(op)
    wb, wp = oracle.hash_join(abi.ColView(bk.ctypes.data, abi.T_I64, 0, 0, 0), len(bk),
                              abi.ColView(pk.ctypes.data, abi.T_I64, 0, 0, 0), len(pk))
    assert m == len(wb)
    for p in range(P):  # pairs grouped by probe partition
        seg = gp[outoff[p]:outoff[p + 1] if p + 1 < P else m]
        assert np.all((seg >= poff[p]) & (seg < poff[p + 1]))
    g, w = np.lexsort((gb, gp)), np.lexsort((wb, wp))
    assert np.array_equal(gp[g], wp[w]) and np.array_equal(gb[g], wb[w])
