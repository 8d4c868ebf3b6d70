"""Synthetic tables and queries of the benchmark workloads (seeded; no public dataset is used).

Tables are cut into segments of 2^20 rows as the engine stores them (src/storage.h:33).  A column is
raw, or encoded in the engine's segment format (src/storage.cu:1138-1192): a 16-byte header holding the
int64 base, then uint8 / uint16 / uint32 offsets from it (the all-ones code is NULL), padded by 16
bytes.  Every segment column is its own 256-byte aligned region of one device allocation per column.

Workloads (sizes as benchmarked):
  * filter_groupby_1m: 2^20 rows; k int32 U[0,16), v int64 U[0,1e6), f float64 U[0,1);
    WHERE v < 500000 GROUP BY k: COUNT(*), SUM(v), MIN(v), MAX(v), AVG(f)  (hash GROUP BY).
  * pricing_summary_60m: 60,000,000 rows; ship_date int32 U[0,2557); quantity int64 U[1,50];
    price int64 cents U[90000,10500000]; discount int64 U[0,10]; tax int64 U[0,8]; flag1 / flag2 uint8
    dictionary codes U[0,3) / U[0,2) stored as 1-byte encoded columns; WHERE ship_date <= 2467
    GROUP BY flag1, flag2 (dense, 6 groups): COUNT(*), SUM(quantity), SUM(price),
    SUM(price*(100-discount)), SUM(price*(100-discount)*(100+tax)), AVG(quantity), AVG(price),
    AVG(discount), all integer sums exact (int128).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import query as q

SEG_ROWS = 1 << 20
ALIGN = 256


def encode_for(x: np.ndarray, width: int, null=None) -> tuple[np.ndarray, int]:
    """Frame-of-reference encoding (enc 1/2/3 = width 1/2/4): (header + codes + 16 pad bytes, base)."""
    valid = x if null is None else x[x != null]
    base = int(valid.min()) if valid.size else 0
    codes = (x.astype(np.int64) - base)
    top = (1 << (8 * width)) - 1
    if valid.size and int(valid.max()) - base >= top:
        raise ValueError("range too wide for this width")
    if null is not None:
        codes = np.where(x == null, top, codes)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32}[width]
    out = np.zeros(16 + x.size * width + 16, dtype=np.uint8)
    out[:8] = np.frombuffer(np.int64(base).tobytes(), dtype=np.uint8)
    out[16:16 + x.size * width] = np.frombuffer(codes.astype(dt).tobytes(), dtype=np.uint8)
    return out, base


def encode_bitpack(x: np.ndarray, null=None) -> np.ndarray:
    """Bit-packed segment column (enc 7): header [int64 base][int32 bits][int32 0], codes x - base in
    `bits` bits each, LSB-first in little-endian 32-bit words, the all-ones code for NULL, 16 pad bytes."""
    x = x.astype(np.int64)
    isnull = (x == null) if null is not None else np.zeros(x.size, bool)
    valid = x[~isnull]
    base = int(valid.min()) if valid.size else 0
    rng = (int(valid.max()) - base) if valid.size else 0
    b = 1
    while (rng + 1) >> b:
        b += 1
    if b > 32:
        raise ValueError("range too wide to bit-pack")
    mask = (1 << b) - 1
    codes = np.where(isnull, mask, x - base).astype(np.uint64)
    nwords = (x.size * b + 31) // 32
    words = np.zeros(nwords + 4, dtype=np.uint64)
    start = np.arange(x.size, dtype=np.uint64) * np.uint64(b)
    w, sh = (start >> np.uint64(5)).astype(np.int64), start & np.uint64(31)
    np.bitwise_or.at(words, w, (codes << sh) & np.uint64(0xFFFFFFFF))
    spill = (sh + np.uint64(b)) > np.uint64(32)
    np.bitwise_or.at(words, w[spill] + 1, codes[spill] >> (np.uint64(32) - sh[spill]))
    out = np.zeros(16 + 4 * nwords + 16, dtype=np.uint8)
    out[:8] = np.frombuffer(np.int64(base).tobytes(), np.uint8)
    out[8:12] = np.frombuffer(np.int32(b).tobytes(), np.uint8)
    out[16:16 + 4 * nwords] = np.frombuffer(words[:nwords].astype(np.uint32).tobytes(), np.uint8)
    return out


def encode_rle(x: np.ndarray) -> np.ndarray:
    """Run-length segment column (enc 8): header [int64 runs][int64 0], int32 exclusive run ends
    (padded to 8 bytes), int64 run values (NULL sentinels included), 16 pad bytes."""
    x = x.astype(np.int64)
    starts = np.flatnonzero(np.concatenate([[True], x[1:] != x[:-1]])) if x.size else np.zeros(0, np.int64)
    runs = starts.size
    ends = np.concatenate([starts[1:], [x.size]]).astype(np.int32) if runs else np.zeros(0, np.int32)
    eb = (runs * 4 + 7) & ~7
    out = np.zeros(16 + eb + 8 * runs + 16, dtype=np.uint8)
    out[:8] = np.frombuffer(np.int64(runs).tobytes(), np.uint8)
    out[16:16 + 4 * runs] = np.frombuffer(ends.tobytes(), np.uint8)
    out[16 + eb:16 + eb + 8 * runs] = np.frombuffer(x[starts].tobytes(), np.uint8)
    return out


@dataclass
class Column:
    name: str
    t: int                 # view type (abi.T_*)
    data: np.ndarray       # host values (full table)
    enc: int = 0           # 0 raw, 1/2/3 encoded (uint8/16/32), 7 bit-packed, 8 run-length
    scale: int = 0
    seg_bytes: list = field(default_factory=list)   # per segment: host bytes of the stored segment column
    host: np.ndarray | None = None                   # all segments' bytes back to back (aligned)
    offsets: list = field(default_factory=list)      # byte offset of each segment in `host`
    dev = None                                       # DeviceBuffer mirror of `host`


class Table:
    """A table of equally segmented columns with host and device copies."""

    def __init__(self, n: int, seg_rows: int = SEG_ROWS):
        self.n = n
        self.seg_rows = seg_rows
        self.cols: list[Column] = []
        self.nseg = (n + seg_rows - 1) // seg_rows

    def seg_len(self, s: int) -> int:
        return min(self.seg_rows, self.n - s * self.seg_rows)

    def add(self, name: str, t: int, data: np.ndarray, enc: int = 0, scale: int = 0) -> int:
        c = Column(name, t, data, enc, scale)
        width = {1: 1, 2: 2, 3: 4}.get(enc, data.dtype.itemsize)
        null = None
        if t in (abi.T_I32N,):
            null = abi.NULL_I32
        elif t in (abi.T_I64N, abi.T_DEC):
            null = abi.NULL_I64
        off = 0
        for s in range(self.nseg):
            lo, hi = s * self.seg_rows, min(self.n, (s + 1) * self.seg_rows)
            if enc == 7:
                b = encode_bitpack(data[lo:hi], null)
            elif enc == 8:
                b = encode_rle(data[lo:hi])
            elif enc:
                b, _ = encode_for(data[lo:hi], width, null)
            else:
                b = np.frombuffer(np.ascontiguousarray(data[lo:hi]).tobytes(), dtype=np.uint8)
            c.seg_bytes.append(b)
            c.offsets.append(off)
            off += (b.size + ALIGN - 1) // ALIGN * ALIGN
        host = np.zeros(max(off, 1), dtype=np.uint8)
        for s, b in enumerate(c.seg_bytes):
            host[c.offsets[s]:c.offsets[s] + b.size] = b
        c.host = host
        c.seg_bytes = []
        self.cols.append(c)
        return len(self.cols) - 1

    def to_device(self):
        from .ops import DeviceBuffer
        for c in self.cols:
            if c.dev is None:
                c.dev = DeviceBuffer.from_array(c.host)

    def free_device(self):
        for c in self.cols:
            if c.dev is not None:
                c.dev.free()
                c.dev = None

    def views(self, s: int, device: bool) -> list:
        vs = []
        for c in self.cols:
            base = c.dev.ptr if device else c.host.ctypes.data
            vs.append(abi.ColView(base + c.offsets[s], c.t, c.scale, c.enc, 0))
        return vs

    def batches(self, device: bool, deleted: list | None = None) -> list:
        """[(rows, deleted bitmap ptr, views)] per segment."""
        return [(self.seg_len(s), deleted[s] if deleted else 0, self.views(s, device)) for s in range(self.nseg)]

    def nbytes(self) -> int:
        return int(sum(c.host.size for c in self.cols))


def env_for(table: Table) -> q.Env:
    """An Env with one slot per table column (slot i = column i), carrying the types and encoding hints."""
    e = q.Env()
    for c in table.cols:
        e.column(c.t, c.scale, c.enc)
    return e


# ------------------------------------------------------------------ filter + GROUP BY, 1M rows
def filter_groupby_1m(n: int = 1 << 20, seed: int = 0) -> Table:
    rng = np.random.default_rng(seed)
    t = Table(n)
    t.add("k", abi.T_I32, rng.integers(0, 16, n, dtype=np.int32))
    t.add("v", abi.T_I64, rng.integers(0, 1_000_000, n, dtype=np.int64))
    t.add("f", abi.T_F64, rng.random(n))
    return t


def filter_groupby_1m_query(table: Table):
    e = env_for(table)
    k, v, f = 0, 1, 2
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(v), "BIGINT", True), q.Agg("MIN", q.col(v), "BIGINT", True),
            q.Agg("MAX", q.col(v), "BIGINT", True), q.Agg("AVG", q.col(f), "DOUBLE", True)]
    aq = q.AggQuery(e, q.col(v).lt(500_000), [(q.col(k), True)], aggs)
    return e, aq


# ------------------------------------------------------------------ pricing summary, 60M rows
PRICING_ROWS = 60_000_000


def pricing_summary(n: int = PRICING_ROWS, seed: int = 2) -> Table:
    rng = np.random.default_rng(seed)
    t = Table(n)
    t.add("ship_date", abi.T_I32, rng.integers(0, 2557, n, dtype=np.int32))
    t.add("quantity", abi.T_I64, rng.integers(1, 51, n, dtype=np.int64))
    t.add("price", abi.T_I64, rng.integers(90_000, 10_500_001, n, dtype=np.int64))
    t.add("discount", abi.T_I64, rng.integers(0, 11, n, dtype=np.int64))
    t.add("tax", abi.T_I64, rng.integers(0, 9, n, dtype=np.int64))
    t.add("flag1", abi.T_I32, rng.integers(0, 3, n, dtype=np.int32), enc=1)
    t.add("flag2", abi.T_I32, rng.integers(0, 2, n, dtype=np.int32), enc=1)
    return t


def pricing_summary_query(table: Table, cutoff: int = 2467):
    e = env_for(table)
    ship, qty, price, disc, tax, f1, f2 = range(7)
    dp = q.col(price) * (q.ilit(100) - q.col(disc))
    ch = dp * (q.ilit(100) + q.col(tax))
    aggs = [q.Agg("COUNT"), q.Agg("SUM", q.col(qty), "BIGINT", True), q.Agg("SUM", q.col(price), "BIGINT", True),
            q.Agg("SUM", dp, "BIGINT", False), q.Agg("SUM", ch, "BIGINT", False),
            q.Agg("AVG", q.col(qty), "BIGINT", True), q.Agg("AVG", q.col(price), "BIGINT", True),
            q.Agg("AVG", q.col(disc), "BIGINT", True)]
    aq = q.AggQuery(e, q.col(ship).le(cutoff), [(q.col(f1), True), (q.col(f2), True)], aggs)
    ds = q.dense_spec(aq.plan, [(0, 2), (0, 1)], table.n)
    return e, aq, ds


# bytes each workload reads per row (the roofline's algorithmic bytes)
PRICING_BYTES_PER_ROW = 4 + 8 * 4 + 1 + 1
FILTER_GROUPBY_BYTES_PER_ROW = 4 + 8 + 8


# ------------------------------------------------------------------ hash join + aggregate
JOIN_BUILD_ROWS = 15_000_000
JOIN_PROBE_ROWS = 60_000_000
JOIN_GROUP_KEYS = 1 << 20
# build: key 8 + order_date 4; probe: fk 8 + cents 8 + gkey 4
JOIN_BUILD_BYTES_PER_ROW = 12
JOIN_PROBE_BYTES_PER_ROW = 20


def join_tables(nb: int = JOIN_BUILD_ROWS, np_: int = JOIN_PROBE_ROWS, seed: int = 3):
    """orders (build): key int64 = a permutation of [0, nb), order_date int32 U[0, 2406);
    lineitem (probe): fk int64 U[0, nb), cents int64 U[0, 1e6), gkey int32 U[0, 2^20)."""
    rng = np.random.default_rng(seed)
    build = Table(nb)
    build.add("key", abi.T_I64, rng.permutation(nb).astype(np.int64))
    build.add("order_date", abi.T_I32, rng.integers(0, 2406, nb, dtype=np.int32))
    probe = Table(np_)
    probe.add("fk", abi.T_I64, rng.integers(0, nb, np_, dtype=np.int64))
    probe.add("cents", abi.T_I64, rng.integers(0, 1_000_000, np_, dtype=np.int64))
    probe.add("gkey", abi.T_I32, rng.integers(0, JOIN_GROUP_KEYS, np_, dtype=np.int32))
    return build, probe


def contiguous_view(t: Table, c: int, device: bool) -> abi.ColView:
    """One view over all rows of a raw column (its segments lie back to back)."""
    col = t.cols[c]
    w = col.data.dtype.itemsize
    assert col.enc == 0 and all(col.offsets[s] == s * t.seg_rows * w for s in range(t.nseg))
    return abi.ColView(col.dev.ptr if device else col.host.ctypes.data, col.t, 0, 0, 0)


def join_aggregate_plans(cutoff: int = 1203):
    """(build filter env + program, aggregation env + AggQuery + DenseSpec over the joined rows)."""
    eb = q.Env()
    eb.column(abi.T_I64)
    eb.column(abi.T_I32)
    where = eb.compile(q.col(1).lt(cutoff))
    ej = q.Env()
    gk = ej.column(abi.T_I32)
    ct = ej.column(abi.T_I64)
    aq = q.AggQuery(ej, None, [(q.col(gk), True)], [q.Agg("COUNT"), q.Agg("SUM", q.col(ct), "BIGINT", True)])
    ds = q.dense_spec(aq.plan, [(0, JOIN_GROUP_KEYS - 1)], JOIN_PROBE_ROWS)
    return eb, where, ej, aq, ds


def join_aggregate_run(build: Table, probe: Table, plans, timer=None):
    """The engine's join pipeline on the device: select build rows (order_date < cutoff), gather their
    keys, inner hash join with the probe keys, gather the probe's gkey and cents for the pairs, dense
    GROUP BY gkey: COUNT, SUM(cents).  timer(name) -> context manager timing a stage.
    Returns (keys, accs in the engine format, pairs)."""
    import contextlib

    from . import ops
    eb, where, ej, aq, ds = plans
    timer = timer or (lambda name: contextlib.nullcontext())
    build.to_device()
    probe.to_device()
    keyv = contiguous_view(build, 0, True)
    fkv = contiguous_view(probe, 0, True)
    ops.jit_set_mode(abi.JIT_SYNC)
    fp = abi.AggPlan()
    fp.hasWhere, fp.where, fp.naggs = 1, where, 1
    fp.ops[0] = abi.AGG_COUNT
    fprog = ops.jit_get(eb.env, eb.ncols, fp, abi.JF_FLAGM, "join build filter")
    aprog = ops.jit_get(ej.env, ej.ncols, aq.plan, abi.JF_DENSE, "join aggregate")
    with timer("select"):
        idx, mb, _ = ops.select_multi(eb.env, where, build.batches(True), eb.ncols, fprog)
    bkeys = ops.DeviceBuffer(max(mb, 1) * 8)
    with timer("gather build keys"):
        ops.gather(keyv.p, abi.PT_I64, idx, mb, bkeys.ptr)
    with timer("join"):
        ob, op, m = ops.hash_join(abi.ColView(bkeys.ptr, abi.T_I64, 0, 0, 0), mb, fkv, probe.n)
    gk, ct = ops.DeviceBuffer(max(m, 1) * 4), ops.DeviceBuffer(max(m, 1) * 8)
    with timer("gather probe columns"):
        ops.gather(probe.cols[2].dev.ptr, abi.PT_I32, op, m, gk.ptr)
        ops.gather(probe.cols[1].dev.ptr, abi.PT_I64, op, m, ct.ptr)
    with timer("aggregate"):
        agg = ops.GpuAggregator(aq.plan, 1024, ds)
        agg.add_batches(ej.ncols, [(m, 0, [abi.ColView(gk.ptr, abi.T_I32, 0, 0, 0),
                                           abi.ColView(ct.ptr, abi.T_I64, 0, 0, 0)])])
        agg.run(ej.env, aprog)
        keys, accs, _ = agg.fetch(exact=False)
    agg.close()
    for p in (idx, ob, op):
        ops.tmp_free(p)
    ops.jit_set_mode(-1)
    return keys, accs, m


# ---------------------------------------------------------------- high-cardinality GROUP BY
# 100,000,000 rows; key int64 = a bijective 64-bit mix of a Zipf(s=1.1) rank over 10,000,000 ranks
# (sparse keys, so the engine hashes rather than indexing dense arrays); payload int64 U[0, 1e9);
# s int32 dictionary codes U[0, 5,000,000) (a string column's codes); WHERE payload < c (c drawn from
# the seed) GROUP BY key: COUNT(*), SUM(payload) [, COUNT(DISTINCT s)].
HC_ROWS = 100_000_000
HC_RANKS = 10_000_000
HC_DICT = 5_000_000
HC_ZIPF_S = 1.1
HC_BYTES_PER_ROW = 16  # key + payload (the distinct pass also reads s: 20)


def zipf_ranks(rng: np.random.Generator, n: int, nranks: int, s: float) -> np.ndarray:
    """n draws of a rank in [0, nranks) with P(r) proportional to (r + 1)^-s (inverse CDF)."""
    w = np.arange(1, nranks + 1, dtype=np.float64) ** -s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    out = np.empty(n, dtype=np.int64)
    step = 1 << 24
    for lo in range(0, n, step):  # bounded temporaries
        hi = min(n, lo + step)
        out[lo:hi] = np.searchsorted(cdf, rng.random(hi - lo), side="right")
    np.minimum(out, nranks - 1, out=out)
    return out


def mix64_np(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer over uint64 (a bijection)."""
    z = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def high_cardinality(n: int = HC_ROWS, nranks: int = HC_RANKS, ndict: int = HC_DICT, seed: int = 4) -> Table:
    rng = np.random.default_rng(seed)
    ranks = zipf_ranks(rng, n, nranks, HC_ZIPF_S)
    key = mix64_np(ranks.astype(np.uint64) + np.uint64(seed * 0x9E3779B9 + 1)).view(np.int64)
    key[key == abi.NULL_I64] += 1  # never the BIGINT NULL sentinel
    del ranks
    t = Table(n)
    t.add("key", abi.T_I64, key)
    t.add("payload", abi.T_I64, rng.integers(0, 1_000_000_000, n, dtype=np.int64))
    t.add("s", abi.T_I32, rng.integers(0, ndict, n, dtype=np.int32))
    return t


def high_cardinality_cut(seed: int = 4) -> int:
    """The predicate constant c of `payload < c` for a run (selectivity 30%..90%)."""
    return int(np.random.default_rng(seed + 1000).integers(300_000_000, 900_000_001))


def high_cardinality_query(t: Table, cut: int, distinct: bool = False):
    """(env, AggQuery, distinct program or None): GROUP BY key COUNT(*), SUM(payload)."""
    e = env_for(t)
    aq = q.AggQuery(e, q.col(1).lt(cut), [(q.col(0), True)], [q.Agg("COUNT"), q.Agg("SUM", q.col(1), "BIGINT", True)],
                    distinct=distinct)
    dprog = e.compile(q.col(2)) if distinct else None
    return e, aq, dprog


def plain_capacity(plan: abi.AggPlan, est: int) -> int:
    """The engine's hash table capacity for an estimate of the group count: pow2 >= 2 est, at least
    1024, the table kept <= 1 GiB (src/engine_select.cpp:1230-1235)."""
    cap = 1024
    max_cap = (1 << 30) // (8 + 8 * plan.nkeys + 8 * plan.naggs)
    while cap < est * 2 and cap * 2 <= max_cap:
        cap <<= 1
    return cap


def grow_capacity(cap: int, groups: int) -> int:
    """Capacity after an overflow: pow2 >= max(4 cap, 4 groups) (src/engine_select.cpp:1514-1522)."""
    want = max(cap * 4, groups * 4)
    c = 1
    while c < want:
        c <<= 1
    return c


def hash_aggregate_run(batches: list, e, aq, cap: int, jit=None):
    """GROUP BY over device batches with the engine's overflow retry: (keys, accs engine format,
    final capacity, runs)."""
    from . import ops
    runs = 0
    while True:
        runs += 1
        agg = ops.GpuAggregator(aq.plan, cap)
        agg.add_batches(e.ncols, batches)
        agg.run(e.env, jit)
        if agg.overflowed():
            g = agg.group_count()
            agg.close()
            cap = grow_capacity(cap, g)
            continue
        keys, accs, _ = agg.fetch(exact=False)
        agg.close()
        return keys, accs, cap, runs


def distinct_plans(e, aq, dprog, dist_int: bool = True):
    """Phase-1 plan of COUNT(DISTINCT x): the plan's keys plus x, every aggregate as a partial per
    (keys, x) (src/engine_select.cpp:1404-1409)."""
    p1 = abi.AggPlan()
    ctypes.memmove(ctypes.byref(p1), ctypes.byref(aq.plan), ctypes.sizeof(abi.AggPlan))
    nk = aq.plan.nkeys
    p1.nkeys = nk + 1
    p1.keys[nk] = dprog
    p1.keyInt[nk] = 1 if dist_int else 0
    p1.densePriv = 0
    return p1


def distinct_phase2(plan: abi.AggPlan, p1: abi.AggPlan, keys_ptr: int, accs_ptr: int, g1: int, dist_int: bool = True):
    """Phase 2 over the compacted (keys, x) groups (column-major device arrays): GROUP BY the keys,
    COUNT / SUM partials summed, MIN by MIN, MAX by MAX, plus one slot counting the pairs whose x is
    not NULL (src/engine_select.cpp:1436-1470).  Returns (env2, ncols2, plan2)."""
    nk, na = plan.nkeys, p1.naggs
    env2 = abi.ExprEnv()
    nc = 0
    for k in range(nk + 1):
        is_int = (plan.keyInt[k] != 0) if k < nk else dist_int
        env2.cols[k] = abi.ColView(keys_ptr + k * g1 * 8, abi.T_I64 if is_int else abi.T_F64, 0, 0, 0)
        env2.code[nc] = abi.Instr(abi.OP_COL, 1 if is_int else 0, k)
        nc += 1
    p2 = abi.AggPlan()
    p2.nkeys = nk
    for k in range(nk):
        p2.keys[k] = abi.Prog(k, 1)
        p2.keyInt[k] = plan.keyInt[k]
    for a in range(na):
        env2.cols[nk + 1 + a] = abi.ColView(accs_ptr + a * g1 * 8, abi.T_I64 if p1.aggBits[a] else abi.T_F64, 0, 0, 0)
        p2.aggs[a] = abi.Prog(nc, 1)
        env2.code[nc] = abi.Instr(abi.OP_COL, 0, nk + 1 + a)
        nc += 1
        p2.ops[a] = abi.AGG_SUM if p1.ops[a] == abi.AGG_COUNT else p1.ops[a]
        p2.aggInt[a] = p2.aggBits[a] = p1.aggBits[a]
        p2.aggPart[a] = 0
    if dist_int:
        p2.aggs[na] = abi.Prog(nc, 1)
        env2.code[nc] = abi.Instr(abi.OP_CONST, 0, 0)
        env2.consts[0] = 1.0
        nc += 1
    else:
        p2.aggs[na] = abi.Prog(nc, 3)
        env2.code[nc] = abi.Instr(abi.OP_COL, 0, nk)
        env2.code[nc + 1] = abi.Instr(abi.OP_ISNULL, 0, 0)
        env2.code[nc + 2] = abi.Instr(abi.OP_NOT, 0, 0)
        nc += 3
    p2.ops[na] = abi.AGG_SUM
    p2.aggInt[na] = 0
    p2.naggs = na + 1
    return env2, nk + 1 + na, p2


def distinct_aggregate_run(batches: list, e, aq, dprog, rows_in: int, timer=None, sizing: str = "plain"):
    """GROUP BY keys with COUNT(DISTINCT x) as the engine runs it: phase 1 hash GROUP BY (keys, x)
    with capacity pow2 >= min(rows, 2^22) and the overflow retry, compaction on the device, phase 2
    GROUP BY keys over the distinct pairs (src/engine_select.cpp:1397-1492).  Returns (keys, accs in
    the engine format with the distinct count as the last slot, phase-1 runs, distinct pairs).
    sizing "learned": the phase-1 table is sized from the estimator's prediction of the
    pair count instead (estimator.py), the plain overflow retry remaining the fallback."""
    import contextlib

    from . import ops
    timer = timer or (lambda name: contextlib.nullcontext())
    p1 = distinct_plans(e, aq, dprog)
    cap1 = 1024
    while cap1 < min(max(rows_in, 1), 1 << 22):
        cap1 <<= 1
    runs = 0
    ops.jit_set_mode(abi.JIT_SYNC)
    try:
        jit1 = ops.jit_get(e.env, e.ncols, p1, abi.JF_GROUPED, "aggregate (distinct pairs)")
        with timer("phase 1 (keys, x)"):
            if sizing == "learned":
                from . import estimator
                cap1 = estimator.learned_capacity(estimator.estimate_groups(e.env, e.ncols, p1, batches))
            while True:
                runs += 1
                a1 = ops.GpuAggregator(p1, cap1)
                a1.add_batches(e.ncols, batches)
                a1.run(e.env, jit1)
                if a1.overflowed():
                    g = a1.group_count()
                    a1.close()
                    cap1 = grow_capacity(cap1, g)
                    continue
                kp, ap, g1 = a1.compact()
                a1.close()
                break
        with timer("phase 2 (keys)"):
            env2, nc2, p2 = distinct_phase2(aq.plan, p1, kp, ap, g1)
            cap2 = 1024
            while cap2 < 2 * g1:
                cap2 <<= 1
            jit2 = ops.jit_get(env2, nc2, p2, abi.JF_GROUPED, "count distinct")
            a2 = ops.GpuAggregator(p2, cap2)
            a2.add_batches(nc2, [(g1, 0, [env2.cols[c] for c in range(nc2)])])
            a2.run(env2, jit2)
            if a2.overflowed():
                raise RuntimeError("phase 2 overflowed a table of twice the pair count")
            keys, accs, _ = a2.fetch(exact=False)
            a2.close()
        ops.tmp_free(kp)
        ops.tmp_free(ap)
    finally:
        ops.jit_set_mode(-1)
    return keys, accs, runs, g1
