"""The TMA-staged scan (tile stages brought into shared memory by bulk copies, a producer warp and
full / empty mbarriers; compiled plans with WARPSTORE_B200_STAGES >= 2): parity with the oracle for the
no-key and private-row GROUP BY scans (ragged batches, a deleted bitmap, an encoded key), and its
bounded waits: with a wait limit far below a copy's latency every wait runs out, the call returns the
staged-copy error instead of a result, and the next call on the same context succeeds.  Each case runs
in a child process because the settings are read once per process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PARITY = r"""
import numpy as np
from oracle import oracle
from warpstore_b200 import abi, ops
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W
from tests.helpers import compare_exact

ops.gpu_init()
rng = np.random.default_rng(31)
n = 3 * (1 << 18) + 12_345                         # ragged last batch
t = W.Table(n, seg_rows=1 << 18)
t.add("d", abi.T_I32, rng.integers(0, 2557, n, dtype=np.int32))
t.add("p", abi.T_I64, rng.integers(90_000, 10_500_001, n, dtype=np.int64))
t.add("x", abi.T_I64, rng.integers(0, 11, n, dtype=np.int64))
t.add("f", abi.T_I32, rng.integers(0, 3, n, dtype=np.int32), enc=1)
t.add("g", abi.T_I32, rng.integers(0, 2, n, dtype=np.int32))
t.to_device()
deleted = []
dev_del = []
for s in range(t.nseg):
    words = (t.seg_len(s) + 31) // 32
    bits = rng.integers(0, 2**32, words, dtype=np.uint64).astype(np.uint32) & np.uint32(0x01010101)
    deleted.append(bits)
    dev_del.append(ops.DeviceBuffer.from_array(bits))
hb = t.batches(False, [d.ctypes.data for d in deleted])
db = t.batches(True, [d.ptr for d in dev_del])
ops.jit_set_mode(abi.JIT_SYNC)
runs = 0
for keys in ([], [(q.col(3), True), (q.col(4), True)]):
    e = W.env_for(t)
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(1) * (q.ilit(100) - q.col(2)), "BIGINT", False),
            q.Agg("MIN", q.col(1), "BIGINT", True), q.Agg("MAX", q.col(2), "BIGINT", True)]
    aq = q.AggQuery(e, q.col(0).le(2000), keys, aggs)
    ds = q.dense_spec(aq.plan, [(0, 2), (0, 1)], n) if keys else None
    fn = abi.JF_DENSE if keys else abi.JF_NOKEYS
    prog = ops.jit_get(e.env, e.ncols, aq.plan, fn, "staged")
    assert prog and ops.jit_info(prog).state == 1
    agg = ops.GpuAggregator(aq.plan, 1024, ds)
    agg.add_batches(e.ncols, db)
    agg.run(e.env, prog)
    k, a, ex = agg.fetch()
    agg.close()
    ok, ow, _ = oracle.aggregate(e.env, aq.plan, hb, e.ncols)
    compare_exact(aq.plan, k, ex, ok, ow)
    runs += 1
print("OK", runs, ops.kernel_launches())
"""

TIMEOUT = r"""
import numpy as np
from warpstore_b200 import abi, ops
from warpstore_b200 import workloads as W

ops.gpu_init()
t = W.pricing_summary(4 * (1 << 20), seed=2)
e, aq, ds = W.pricing_summary_query(t)
t.to_device()
ops.jit_set_mode(abi.JIT_SYNC)
prog = ops.jit_get(e.env, e.ncols, aq.plan, abi.JF_DENSE, "staged")
agg = ops.GpuAggregator(aq.plan, 1024, ds)
agg.add_batches(e.ncols, t.batches(True))
try:
    agg.run(e.env, prog)
    agg.fetch()
    print("NO ERROR")
except ops.WsError as err:
    print("ERROR", err.code, err)
agg.close()
# the context stays usable: a plain device round trip after the reported error
b = ops.DeviceBuffer.from_array(np.arange(1000, dtype=np.int64))
assert int(b.to_array(np.int64).sum()) == 499500
print("CONTEXT OK")
"""


def run_child(code, **env):
    e = dict(os.environ, **env)
    r = subprocess.run([sys.executable, "-c", code], env=e, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return r.stdout.strip().splitlines()


@pytest.mark.parametrize("stages", ["2", "3"])
def test_staged_scans_match_the_oracle(stages):
    out = run_child(PARITY, WARPSTORE_B200_STAGES=stages)
    assert out[-1].startswith("OK 2")


def test_staged_wait_limit_reports_an_error_and_the_context_survives():
    out = run_child(TIMEOUT, WARPSTORE_B200_STAGES="3", WARPSTORE_B200_WAIT_LIMIT_LOG2="4")
    assert out[-1] == "CONTEXT OK"
    assert out[-2].startswith("ERROR 1105") and "staged" in out[-2], out
