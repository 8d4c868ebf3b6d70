"""Hash join + aggregate (the engine's join pipeline: select build rows, gather keys, inner hash join,
gather probe columns, dense GROUP BY) through this library's operators, checked against the CPU oracle
(row-exact groups) and against the same pipeline on the reference's own operators."""
import time
from contextlib import contextmanager

import numpy as np
import pytest
import torch

from oracle import oracle, ref
from warpstore_b200 import abi
from warpstore_b200 import workloads as W

from . import ref_pipelines as RP
from .tests_join_util import oracle_join_aggregate

pytestmark = pytest.mark.gpu


def engine_groups(aq, keys, accs):
    """{gkey: (count, exact sum)} from the engine format (split BIGINT sum recombined)."""
    a_sum = aq.aggs[1]
    bits = accs.view(np.int64)
    kk = keys.view(np.int64)[:, 0]
    out = {}
    for i in range(accs.shape[0]):
        s = int(bits[i, a_sum.hi_slot]) * (1 << 32) + int(bits[i, a_sum.slot])
        out[int(kk[i])] = (int(accs[i, 0]), s)
    return out


def test_join_aggregate_matches_oracle_and_reference():
    build, probe = W.join_tables(1_500_000, 6_000_000, seed=5)
    plans = W.join_aggregate_plans()
    keys, accs, m = W.join_aggregate_run(build, probe, plans)
    got = engine_groups(plans[3], keys, accs)
    want, wm = oracle_join_aggregate(build, probe, plans)
    assert m == wm
    assert got == want
    if ref.available():
        rk, ra, rm = RP.join_aggregate_run(build, probe, plans)
        assert rm == m and engine_groups(plans[3], rk, ra) == got


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_join_aggregate_full_size_vs_oracle_and_reference():
    build, probe = W.join_tables()
    plans = W.join_aggregate_plans()
    times = {}

    def timer_for(impl):
        """Wall clock with the device synchronized on both sides: the stages mix kernels with host work
        (result downloads into pageable memory), which CUDA events alone would not see."""
        @contextmanager
        def t(name):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            yield
            torch.cuda.synchronize()
            times[(impl, name)] = 1e3 * (time.perf_counter() - t0)
        return t

    runners = {"ours": W.join_aggregate_run, "reference": RP.join_aggregate_run}
    res = {}
    for impl in ("ours", "reference"):
        runners[impl](build, probe, plans)  # warm (plans compiled, pools grown)
        res[impl] = runners[impl](build, probe, plans, timer_for(impl))
    got = engine_groups(plans[3], *res["ours"][:2])
    want, wm = oracle_join_aggregate(build, probe, plans)
    assert res["ours"][2] == wm and got == want
    assert res["ours"][2] == res["reference"][2]
    assert got == engine_groups(plans[3], *res["reference"][:2])
    stages = ["select", "gather build keys", "join", "gather probe columns", "aggregate"]
    print(f"\n[timing] join+aggregate build {build.n} probe {probe.n} pairs {res['ours'][2]}")
    for s in stages:
        print(f"[timing]   {s:22s} reference {times[('reference', s)]:8.3f} ms   ours {times[('ours', s)]:8.3f} ms")
    tr = sum(times[("reference", s)] for s in stages)
    to = sum(times[("ours", s)] for s in stages)
    print(f"[timing]   {'total':22s} reference {tr:8.3f} ms   ours {to:8.3f} ms   ratio {tr / to:.2f}x")
    build.free_device()
    probe.free_device()
