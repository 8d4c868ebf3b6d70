"""The reference's known-answer aggregation queries (tests/golden/known_answers.json, from its
tests/smoke.py) through the GPU operators, compiled and interpreted."""
import numpy as np
import pytest

from warpstore_b200 import abi, ops

from . import known_answers as KA

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", KA.load()["cases"], ids=lambda c: c["name"])
@pytest.mark.parametrize("jit", [True, False], ids=["compiled", "interpreted"])
def test_known_answers_gpu(case, jit):
    g = KA.load()
    st = g["states"][str(case["state"])]
    t = KA.table_of(st)
    t.to_device()
    bset = ops.DeviceBuffer.from_array(np.array([0b0010], dtype=np.uint32))
    e, aq, post = KA.plan_of(case, t, bset.ptr)
    bits = KA.deleted_bits(st)
    dbits = ops.DeviceBuffer.from_array(bits) if bits is not None else None
    fn = abi.JF_NOKEYS if aq.plan.nkeys == 0 else abi.JF_GROUPED
    ops.jit_set_mode(abi.JIT_SYNC if jit else abi.JIT_OFF)
    try:
        prog = ops.jit_get(e.env, e.ncols, aq.plan, fn, case["name"]) if jit else None
        assert (prog is not None) == jit
        agg = ops.GpuAggregator(aq.plan, 1024)
        for i, v in enumerate(t.views(0, True)):
            e.env.cols[i] = v
        agg.add_batch(e.env, e.ncols, t.n, dbits.ptr if dbits else 0)
        agg.run(e.env, prog)
        keys, accs, exact = agg.fetch()
        kb = keys.view(np.int64) if keys.size else np.zeros((exact.shape[0], 0), dtype=np.int64)
        assert KA.result_rows(case, aq, kb, exact, post) == case["expect"]
    finally:
        ops.jit_set_mode(-1)
