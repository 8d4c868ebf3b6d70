"""The reference's known-answer aggregation queries (tests/golden/known_answers.json) as operator plans."""
from __future__ import annotations

import json
import os

import numpy as np

from warpstore_b200 import abi
from warpstore_b200 import query as q
from warpstore_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")


def load():
    return json.load(open(GOLDEN))


def table_of(state: dict) -> W.Table:
    n = len(state["id"])
    t = W.Table(n)
    t.add("id", abi.T_I32, np.array(state["id"], dtype=np.int32))
    t.add("name", abi.T_I32, np.array(state["name"], dtype=np.int32))
    t.add("price", abi.T_F64, np.array(state["price"], dtype=np.float64))
    t.add("d", abi.T_I32, np.array(state["d"], dtype=np.int32))
    return t


def deleted_bits(state: dict) -> np.ndarray | None:
    if not state.get("deleted"):
        return None
    bits = np.zeros((len(state["id"]) + 31) // 32, dtype=np.uint32)
    for r in state["deleted"]:
        bits[r >> 5] |= np.uint32(1) << np.uint32(r & 31)
    return bits


def plan_of(case: dict, t: W.Table, set_ptr: int):
    """(env, AggQuery, post-filter) of a case; set_ptr: bitmap of dictionary codes matching LIKE 'b%'."""
    e = W.env_for(t)
    ID, NAME, PRICE, D = 0, 1, 2, 3
    name = case["name"]
    if name == "group by":
        aq = q.AggQuery(e, None, [(q.col(NAME), True)],
                        [q.Agg("COUNT"), q.Agg("SUM", q.col(PRICE), "DOUBLE", True), q.Agg("MIN", q.col(D), "DATE", True)])
        return e, aq, None
    if name == "or filter":
        s = e.add_set(set_ptr, 4)
        aq = q.AggQuery(e, q.or_(q.inset(q.col(NAME), s), q.col(PRICE).gt(2)), [],
                        [q.Agg("COUNT"), q.Agg("SUM", q.col(PRICE), "DOUBLE", True)])
        return e, aq, None
    if name == "having":
        aq = q.AggQuery(e, None, [(q.col(NAME), True)], [q.Agg("SUM", q.col(PRICE), "DOUBLE", True)])
        return e, aq, lambda row: row[1] > 5
    if name == "case group":
        big = q.select(q.col(PRICE).gt(10), q.ilit(1), q.ilit(0))
        aq = q.AggQuery(e, None, [(big, True)], [q.Agg("COUNT")])
        return e, aq, None
    if name == "year()":
        aq = q.AggQuery(e, None, [(q.year(q.col(D)), True)], [q.Agg("COUNT")])
        return e, aq, None
    raise KeyError(name)


def result_rows(case: dict, aq: q.AggQuery, keys_bits: np.ndarray, words: np.ndarray, post) -> list:
    """SQL result rows (keys, then the case's aggregates) from exact words, sorted by key."""
    rows = []
    for g in range(words.shape[0]):
        row = [int(k) for k in keys_bits[g]] if keys_bits.size else []
        for a in aq.aggs:
            if a.fn == "COUNT":
                row.append(int(words[g, a.slot, 0]))
            elif a.arg_type == "DOUBLE":
                row.append(float(np.array([words[g, a.slot, 0]], dtype=np.int64).view(np.float64)[0]))
            else:
                row.append(int(words[g, a.slot, 0]))
        rows.append(row)
    if post:
        rows = [r for r in rows if post(r)]
    if case["name"] == "having":
        rows.sort(key=lambda r: -r[1])
    else:
        rows.sort()
    return rows
