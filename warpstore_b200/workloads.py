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


@dataclass
class Column:
    name: str
    t: int                 # view type (abi.T_*)
    data: np.ndarray       # host values (full table)
    enc: int = 0           # 0 raw, 1/2/3 encoded (uint8/16/32)
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
            if enc:
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


def join_aggregate_run(build: Table, probe: Table, plans, impl: str = "ours", timer=None):
    """The engine's join pipeline on the device: select build rows (order_date < cutoff), gather their
    keys, inner hash join with the probe keys, gather the probe's gkey and cents for the pairs, dense
    GROUP BY gkey: COUNT, SUM(cents).  impl "ours" runs this library's operators, "reference" the
    reference's (oracle/_ref, tests only).  timer(name) -> context manager timing a stage.
    Returns (keys, accs in the engine format, pairs)."""
    import contextlib

    from . import ops
    eb, where, ej, aq, ds = plans
    timer = timer or (lambda name: contextlib.nullcontext())
    build.to_device()
    probe.to_device()
    keyv = contiguous_view(build, 0, True)
    fkv = contiguous_view(probe, 0, True)
    if impl == "ours":
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
    from oracle import ref  # the reference's operators (test infrastructure)
    with timer("select"):
        idx, mb, _ = ref.select_multi_dev(eb.env, where, build.batches(True), eb.ncols)
    bkeys = ops.DeviceBuffer(max(mb, 1) * 8)
    with timer("gather build keys"):
        ref.gather(keyv.p, abi.PT_I64, idx, mb, bkeys.ptr)
    with timer("join"):
        ob, op, m, _ = ref.hash_join_dev(abi.ColView(bkeys.ptr, abi.T_I64, 0, 0, 0), mb, fkv, probe.n)
    gk, ct = ops.DeviceBuffer(max(m, 1) * 4), ops.DeviceBuffer(max(m, 1) * 8)
    with timer("gather probe columns"):
        ref.gather(probe.cols[2].dev.ptr, abi.PT_I32, op, m, gk.ptr)
        ref.gather(probe.cols[1].dev.ptr, abi.PT_I64, op, m, ct.ptr)
    with timer("aggregate"):
        keys, accs, _, ovf, _ = ref.aggregate(ej.env, ej.ncols, aq.plan,
                                              [(m, 0, [abi.ColView(gk.ptr, abi.T_I32, 0, 0, 0),
                                                       abi.ColView(ct.ptr, abi.T_I64, 0, 0, 0)])], ds, 1024)
    for p in (idx, ob, op):
        ref.free(p)
    return keys, accs, m
