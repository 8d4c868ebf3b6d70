"""The estimator on the GPU: the sketch kernel's registers and counts equal the host definition on the
same sampled rows; the MLP kernel equals the FP32 forward pass over the BF16 weights; learned sizing of
COUNT(DISTINCT)'s phase-1 table gives the plain sizing's result in fewer (or as many) runs."""
import numpy as np
import pytest

from warpstore_b200 import abi, ops
from warpstore_b200 import estimator as E
from warpstore_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table():
    t = W.high_cardinality(3_000_000, 300_000, 200_000, seed=9)
    t.to_device()
    yield t
    t.free_device()


@pytest.mark.parametrize("sample_rows", [1 << 16, 1 << 30], ids=["sampled", "every-row"])
def test_sketch_matches_host_definition(table, sample_rows):
    cut = W.high_cardinality_cut(9)
    e, aq, _ = W.high_cardinality_query(table, cut)
    regs, sampled, passing = E.sketch(e.env, e.ncols, aq.plan, table.batches(True), sample_rows)
    rows = E.sample_rows_of(table.n, sample_rows)
    keys, payload = table.cols[0].data, table.cols[1].data
    mask = payload[rows] < cut
    assert sampled == rows.size and passing == int(mask.sum())
    assert np.array_equal(regs, E.hll_registers(keys[rows][mask].view(np.uint64)))
    if sample_rows > table.n:  # every row: the estimate is within HLL error of the exact count
        exact = np.unique(keys[payload < cut]).size
        assert abs(E.hll_estimate(regs) - exact) / exact < 0.05


def test_mlp_kernel_matches_forward_pass():
    m = E.Model()
    rng = np.random.default_rng(1)
    x = (m.mean + m.std * rng.normal(0, 1, (37, E.NFEATURES))).astype(np.float32)
    np.testing.assert_allclose(m.forward_gpu(x), m.forward_np(x), rtol=2e-4, atol=2e-4)


def test_learned_sizing_same_result_fewer_runs(table):
    e, aq, dprog = W.high_cardinality_query(table, W.high_cardinality_cut(9), distinct=True)
    plain = W.distinct_aggregate_run(table.batches(True), e, aq, dprog, table.n)
    learned = W.distinct_aggregate_run(table.batches(True), e, aq, dprog, table.n, sizing="learned")
    assert learned[3] == plain[3]
    assert learned[2] <= plain[2]
    kp, kl = np.ascontiguousarray(plain[0]).view(np.int64)[:, 0], np.ascontiguousarray(learned[0]).view(np.int64)[:, 0]
    op, ol = np.argsort(kp), np.argsort(kl)
    assert np.array_equal(kp[op], kl[ol])
    assert np.array_equal(plain[1][op].view(np.int64), learned[1][ol].view(np.int64))
    print(f"\n[estimator] distinct pairs {plain[3]}: phase-1 runs plain {plain[2]}, learned {learned[2]}")
