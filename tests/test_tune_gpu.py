"""The launch-shape autotuner on the GPU: in tuning mode the first run of a (scan kernel, plan, size
class) times the candidate shapes on the query's own batches and records the fastest; the result is
the oracle's whatever the shape (the final run starts from reset rows); later runs use the recorded
choice without tuning again; the table persists in the plan-cache directory."""
import os

import pytest

from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

from .helpers import compare_exact
from .test_agg_gpu import gpu_aggregate, oracle_aggregate

pytestmark = pytest.mark.gpu


def run_and_check(t, e, plan, dense=None, cap=1024, jit=True):
    ok, ow, _ = oracle_aggregate(t, e, plan)
    agg = gpu_aggregate(t, e, plan, dense, cap, jit)
    assert not agg.overflowed()
    keys, _, ex = agg.fetch()
    compare_exact(plan, keys, ex, ok, ow)
    agg.close()


@pytest.fixture
def tuning(tmp_path):
    ops.tune_clear()
    ops.jit_set_cache_dir(str(tmp_path))
    ops.tune_set_mode(ops.TUNE_ON)
    yield tmp_path
    ops.tune_set_mode(ops.TUNE_USE)
    ops.jit_set_cache_dir("")
    ops.tune_clear()


def test_tuned_shapes_give_the_oracle_result(tuning):
    t = W.pricing_summary(2_000_000, seed=6)
    e, aq, ds = W.pricing_summary_query(t)
    run_and_check(t, e, aq.plan, ds)                       # dense private rows
    run_and_check(t, e, aq.plan, None, cap=64)             # hash
    run_and_check(t, e, aq.plan, None, cap=64, jit=False)  # hash, interpreted
    e2 = W.env_for(t)
    aq2 = q.AggQuery(e2, q.col(0).le(2467), [], [q.Agg("COUNT"), q.Agg("SUM", q.col(2), "BIGINT", True)])
    run_and_check(t, e2, aq2.plan)                         # no keys
    tab = ops.tune_table()
    kinds = sorted({k.split(":")[0] for k in tab})
    assert kinds == ["dense_priv", "hash", "nokeys"], tab
    assert any(k.split(":")[1].startswith("i") for k in tab)  # the interpreter's own entry
    assert all(us > 0 for *_, us in tab.values())
    # recorded: the same runs tune nothing more
    n = len(tab)
    run_and_check(t, e, aq.plan, ds)
    run_and_check(t, e, aq.plan, None, cap=64)
    assert len(ops.tune_table()) == n
    # persisted next to the compiled plans, and read back
    path = os.path.join(str(tuning), "wsb200_tune.txt")
    lines = open(path).read().splitlines()
    assert len(lines) >= n
    ops.tune_clear()
    ops.jit_set_cache_dir(str(tuning))
    assert set(ops.tune_table()) == set(tab)
    print("\n[tune] " + "; ".join(f"{k.split(':')[0]}: ctas/SM {c or 'max'}, smem {m or 'default'} KB, "
                                  f"stages {'default' if st < 0 else st}, {us:.0f} us"
                                  for k, (c, m, st, _, us) in sorted(tab.items())))


def test_tuned_join_table_gives_the_oracle_pairs(tuning):
    """A sparse-key hash join in tuning mode times 2, 3 and 4 table slots per build key on its own keys,
    records the fastest under its size class and joins with it: the oracle's pairs; a second join of
    the same sizes tunes nothing more."""
    import numpy as np

    from oracle import oracle
    rng = np.random.default_rng(9)
    mul = np.uint64(0x9E3779B97F4A7C15)
    bk = (rng.permutation(4_000_000)[:1_500_000].astype(np.uint64) * mul).view(np.int64)
    pk = (rng.integers(0, 4_000_000, 3_000_000).astype(np.uint64) * mul).view(np.int64)
    db, dp = ops.DeviceBuffer.from_array(bk), ops.DeviceBuffer.from_array(pk)
    bv, pv = abi.ColView(db.ptr, abi.T_I64, 0, 0, 0), abi.ColView(dp.ptr, abi.T_I64, 0, 0, 0)
    for rep in range(2):
        ob, op, m = ops.hash_join(bv, len(bk), pv, len(pk))
        gb, gp = ops.device_to_array(ob, np.int32, m), ops.device_to_array(op, np.int32, m)
        ops.tmp_free(ob)
        ops.tmp_free(op)
        wb, wp = oracle.hash_join(abi.ColView(bk.ctypes.data, abi.T_I64, 0, 0, 0), len(bk),
                                  abi.ColView(pk.ctypes.data, abi.T_I64, 0, 0, 0), len(pk))
        g, w = np.lexsort((gb, gp)), np.lexsort((wb, wp))
        assert m == len(wb) and np.array_equal(gp[g], wp[w]) and np.array_equal(gb[g], wb[w])
        joins = {k: v for k, v in ops.tune_table().items() if k.startswith("join:")}
        assert len(joins) == 1 and list(joins.values())[0][3] in (2, 3, 4)
    print(f"\n[tune] {joins}")
