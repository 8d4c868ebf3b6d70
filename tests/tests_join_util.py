"""CPU oracle of the join + aggregate pipeline (select, join pairs, gathers, GROUP BY)."""
import numpy as np

from oracle import oracle
from warpstore_b200 import abi
from warpstore_b200 import workloads as W


def oracle_join_aggregate(build, probe, plans):
    eb, where, ej, aq, ds = plans
    idx, _ = oracle.select(eb.env, where, build.batches(False), eb.ncols)
    bkeys = np.ascontiguousarray(build.cols[0].data[idx])
    fk = np.ascontiguousarray(probe.cols[0].data)
    ob, op = oracle.hash_join(abi.ColView(bkeys.ctypes.data, abi.T_I64, 0, 0, 0), len(bkeys),
                              abi.ColView(fk.ctypes.data, abi.T_I64, 0, 0, 0), len(fk))
    gk = np.ascontiguousarray(probe.cols[2].data[op])
    ct = np.ascontiguousarray(probe.cols[1].data[op])
    views = [abi.ColView(gk.ctypes.data, abi.T_I32, 0, 0, 0), abi.ColView(ct.ctypes.data, abi.T_I64, 0, 0, 0)]
    keys, words, _ = oracle.aggregate(ej.env, aq.plan, [(len(op), 0, views)], ej.ncols)
    a_sum = aq.aggs[1]
    out = {}
    for i in range(keys.shape[0]):
        lo, hi = words[i, a_sum.slot]
        out[int(keys[i, 0])] = (int(words[i, 0, 0]), int(np.uint64(lo)) + (int(hi) << 64))
    return out, len(op)
