"""The request loop's result digest (no GPU): order-independent over groups, sensitive to every key
bit and exact word, with DOUBLE SUM slots kept apart as a plain total (their last bits depend on the
order of the additions)."""
import numpy as np

from warpstore_b200 import abi
from warpstore_b200 import serving as S


def plan_of_slots(ops, ints, nkeys):
    p = abi.AggPlan()
    p.nkeys, p.naggs = nkeys, len(ops)
    for a, (o, i) in enumerate(zip(ops, ints)):
        p.ops[a], p.aggInt[a] = o, i
    return p


def test_digest_properties():
    rng = np.random.default_rng(0)
    plan = plan_of_slots([abi.AGG_COUNT, abi.AGG_SUM, abi.AGG_MIN, abi.AGG_SUM], [1, 1, 1, 0], 2)
    g = 500
    keys = rng.integers(0, 1 << 20, (g, 2)).astype(np.float64)
    ex = rng.integers(-(1 << 40), 1 << 40, (g, 4, 2)).astype(np.int64)
    ex[:, 3, 0] = rng.random(g).view(np.int64)
    ex[:, 3, 1] = 0
    c, f = S.digest(plan, keys, ex)
    perm = rng.permutation(g)
    c2, f2 = S.digest(plan, keys[perm], ex[perm])
    assert c2 == c and abs(f2 - f) <= 1e-12 * abs(f)
    assert abs(f - ex[:, 3, 0].view(np.float64).sum()) <= 1e-12 * abs(f)
    k3 = keys.copy()
    k3[7, 1] = np.nextafter(k3[7, 1], np.inf)      # one key bit
    assert S.digest(plan, k3, ex)[0] != c
    x3 = ex.copy()
    x3[11, 1, 1] ^= 1                               # the high word of an exact sum
    assert S.digest(plan, keys, x3)[0] != c
    x4 = ex.copy()
    x4[3, 3, 0] = np.array([0.5]).view(np.int64)[0]  # a DOUBLE SUM value: total, not the checksum
    c4, f4 = S.digest(plan, keys, x4)
    assert c4 == c and f4 != f
    assert S.digest(plan, keys[:0], ex[:0]) == (0, 0.0)
