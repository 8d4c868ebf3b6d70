"""Host-side builders of the operator inputs, mirroring what the Warpstore engine hands its GPU layer.

* `Expr` + `Env.compile` emit the engine's stack bytecode into an ExprEnv the way its Compiler does
  (src/engine_core.h:1485-1852): column slots carry the physical type (t) and the encoding hint, integer
  literals keep their int64 bit pattern in the double constant slot, constants are de-duplicated.
* `AggQuery` lays out aggregate slots with the engine's rules (src/engine_select.cpp:647-724 and
  :1130-1149): slot 0 is a hidden COUNT(*); SUM / MIN / MAX share slots by canonical argument; a
  nullable argument gets a non-NULL count slot; with GROUP BY a SUM of a BIGINT column is split into the
  sums of its low and high 32-bit halves (aggPart 1 / 2, exact as int64 bits, aggBits); integer MIN / MAX
  of BIGINT columns keep int64 bits; a nullable integer column argument is read raw (aggNull).
* `dense_spec` builds the DenseSpec of a dense GROUP BY from key ranges with the engine's mode choice
  (src/engine_select.cpp:1172-1229).
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass, field

from . import abi


# Typing of compiled expressions, (ExprEnv, Prog) -> bool.  None: the library's own (ws_prog_is_int).
# A caller timing another implementation of the operators sets its own, so that building the plans
# loads nothing of this library's native code.
TYPER = None


def _i2d(v: int) -> float:
    """The double whose bit pattern is the int64 v (integer literals, src/engine_core.h:1505-1514)."""
    return struct.unpack("<d", struct.pack("<q", v))[0]


class Expr:
    """A bytecode expression tree node."""

    def __init__(self, op: int, kids=(), arg: int = 0, is_int: int = 0, value=None, canon: str = ""):
        self.op, self.kids, self.arg, self.is_int, self.value = op, tuple(kids), arg, is_int, value
        self.canon = canon or f"{op}:{arg}:{is_int}:{value}(" + ",".join(k.canon for k in self.kids) + ")"

    # arithmetic / comparison sugar
    def __add__(self, o): return Expr(abi.OP_ADD, (self, _e(o)))
    def __sub__(self, o): return Expr(abi.OP_SUB, (self, _e(o)))
    def __mul__(self, o): return Expr(abi.OP_MUL, (self, _e(o)))
    def __truediv__(self, o): return Expr(abi.OP_DIV, (self, _e(o)))
    def __mod__(self, o): return Expr(abi.OP_MOD, (self, _e(o)))
    def __neg__(self): return Expr(abi.OP_NEG, (self,))
    def __radd__(self, o): return Expr(abi.OP_ADD, (_e(o), self))
    def __rsub__(self, o): return Expr(abi.OP_SUB, (_e(o), self))
    def __rmul__(self, o): return Expr(abi.OP_MUL, (_e(o), self))
    def eq(self, o): return Expr(abi.OP_EQ, (self, _e(o)))
    def ne(self, o): return Expr(abi.OP_NE, (self, _e(o)))
    def lt(self, o): return Expr(abi.OP_LT, (self, _e(o)))
    def le(self, o): return Expr(abi.OP_LE, (self, _e(o)))
    def gt(self, o): return Expr(abi.OP_GT, (self, _e(o)))
    def ge(self, o): return Expr(abi.OP_GE, (self, _e(o)))


def _e(x) -> Expr:
    if isinstance(x, Expr):
        return x
    if isinstance(x, bool):
        return ilit(int(x))
    if isinstance(x, int):
        return ilit(x)
    return lit(float(x))


def col(slot: int) -> Expr: return Expr(abi.OP_COL, arg=slot)
def colraw(slot: int, is_int: int = 1) -> Expr: return Expr(abi.OP_COLRAW, arg=slot, is_int=is_int)
def ilit(v: int) -> Expr: return Expr(abi.OP_CONST, is_int=1, value=int(v))
def lit(v: float) -> Expr: return Expr(abi.OP_CONST, is_int=0, value=float(v))
def and_(a, b) -> Expr: return Expr(abi.OP_AND, (_e(a), _e(b)))
def or_(a, b) -> Expr: return Expr(abi.OP_OR, (_e(a), _e(b)))
def not_(a) -> Expr: return Expr(abi.OP_NOT, (_e(a),))
def inset(x, set_idx: int) -> Expr: return Expr(abi.OP_INSET, (_e(x),), arg=set_idx)
def select(c, t, e) -> Expr: return Expr(abi.OP_SELECT, (_e(c), _e(t), _e(e)))
def year(x) -> Expr: return Expr(abi.OP_YEAR, (_e(x),))
def isnull(x) -> Expr: return Expr(abi.OP_ISNULL, (_e(x),))
def isnotnull(x) -> Expr: return not_(isnull(x))
def coalesce(a, b) -> Expr: return Expr(abi.OP_COALESCE, (_e(a), _e(b)))
def nullif(a, b) -> Expr: return Expr(abi.OP_NULLIF, (_e(a), _e(b)))
def call1(fn: str, x) -> Expr: return Expr(abi.OP_CALL1, (_e(x),), arg=abi.FN[fn])
def call2(fn: str, a, b) -> Expr: return Expr(abi.OP_CALL2, (_e(a), _e(b)), arg=abi.FN[fn])
def dictmap(x, map_idx: int) -> Expr: return Expr(abi.OP_DICTMAP, (_e(x),), arg=map_idx)
def insorted(x, map_idx: int) -> Expr: return Expr(abi.OP_INSORTED, (_e(x),), arg=map_idx)


class Env:
    """An ExprEnv under construction (one per query)."""

    def __init__(self):
        self.env = abi.ExprEnv()
        self.ncode = 0
        self.nconst = 0
        self.ncols = 0
        self.nsets = 0
        self.nmaps = 0
        self._keep = []  # host buffers referenced by pointers in the env

    def column(self, t: int, scale: int = 0, enc_hint: int = 0) -> int:
        """A column slot of physical view type t (abi.T_*); enc_hint != 0: some segments are encoded."""
        s = self.ncols
        if s >= abi.MAX_COLS:
            raise ValueError("too many columns")
        self.env.cols[s].t = t
        self.env.cols[s].scale = scale
        self.env.cols[s].enc = enc_hint
        self.ncols += 1
        return s

    def add_set(self, dev_ptr: int, nbits: int) -> int:
        i = self.nsets
        self.env.sets[i] = dev_ptr
        self.env.setSize[i] = nbits
        self.nsets += 1
        return i

    def add_map(self, dev_ptr: int, n: int) -> int:
        i = self.nmaps
        self.env.maps[i] = dev_ptr
        self.env.mapSize[i] = n
        self.nmaps += 1
        return i

    def _const(self, e: Expr) -> int:
        bits = _i2d(e.value) if e.is_int else e.value
        raw = struct.pack("<d", bits)
        for i in range(self.nconst):
            if struct.pack("<d", self.env.consts[i]) == raw:
                return i
        if self.nconst >= abi.MAX_CONSTS:
            raise ValueError("too many constants")
        self.env.consts[self.nconst] = bits
        self.nconst += 1
        return self.nconst - 1

    def _emit(self, op: int, arg: int = 0, is_int: int = 0):
        if self.ncode >= abi.MAX_CODE:
            raise ValueError("expression too complex")
        self.env.code[self.ncode] = abi.Instr(op, is_int, arg)
        self.ncode += 1

    def _gen(self, e: Expr):
        for k in e.kids:
            self._gen(k)
        if e.op == abi.OP_CONST:
            self._emit(abi.OP_CONST, self._const(e), e.is_int)
        else:
            self._emit(e.op, e.arg, e.is_int)

    def compile(self, e: Expr) -> abi.Prog:
        start = self.ncode
        self._gen(e)
        return abi.Prog(start, self.ncode - start)

    def is_int(self, prog: abi.Prog) -> bool:
        """Static type of a compiled expression: the library's typing (host only), or TYPER's when set."""
        if TYPER is not None:
            return bool(TYPER(self.env, prog))
        from ._lib import lib
        return bool(lib().ws_prog_is_int(C.byref(self.env), prog))

    def bind(self, slot: int, ptr: int, enc: int = 0, off: int = 0):
        self.env.cols[slot].p = ptr
        self.env.cols[slot].enc = enc
        self.env.cols[slot].off = off

    def views(self) -> list:
        """A copy of the first ncols column views (one batch's views)."""
        return [abi.ColView(self.env.cols[i].p, self.env.cols[i].t, self.env.cols[i].scale, self.env.cols[i].enc,
                            self.env.cols[i].off) for i in range(self.ncols)]


@dataclass
class Agg:
    """One SQL aggregate: fn in COUNT / SUM / MIN / MAX / AVG; arg None = COUNT(*).
    arg_type: BIGINT / INT / DOUBLE / DECIMAL / DATE / DATETIME (the argument's SQL type);
    is_col: the argument is a plain column; nullable: the argument can be NULL."""
    fn: str
    arg: Expr | None = None
    arg_type: str = "BIGINT"
    is_col: bool = False
    nullable: bool = False
    col_slot: int = -1
    slot: int = field(default=-1, init=False)
    hi_slot: int = field(default=-1, init=False)
    cnt_slot: int = field(default=0, init=False)


class AggQuery:
    """Aggregate slots and the AggPlan of one aggregation (engine rules, see module docstring)."""

    def __init__(self, env: Env, where: Expr | None, keys: list, aggs: list[Agg], distinct: bool = False):
        self.env, self.aggs = env, aggs
        plan = abi.AggPlan()
        plan.naggs = 1
        plan.ops[0] = abi.AGG_COUNT
        args = [None]
        by_canon: dict[str, int] = {}
        grouped = bool(keys) or distinct

        def new_slot(op, arg):
            if plan.naggs >= abi.MAX_AGGS:
                raise ValueError("too many aggregates")
            plan.ops[plan.naggs] = op
            args.append(arg)
            plan.naggs += 1
            return plan.naggs - 1

        for a in aggs:
            if a.arg is not None and a.nullable:
                k = "cnt" + a.arg.canon
                if k not in by_canon:
                    by_canon[k] = new_slot(abi.AGG_SUM, isnotnull(a.arg))
                a.cnt_slot = by_canon[k]
            if a.fn == "COUNT":
                a.slot = a.cnt_slot
                continue
            op = abi.AGG_MIN if a.fn == "MIN" else abi.AGG_MAX if a.fn == "MAX" else abi.AGG_SUM
            k = f"{op}:{a.arg.canon}"
            if k not in by_canon:
                s = new_slot(op, a.arg)
                by_canon[k] = s
                if op == abi.AGG_SUM and grouped and a.is_col and a.arg_type in ("BIGINT", "DATETIME"):
                    h = new_slot(abi.AGG_SUM, a.arg)
                    plan.aggPart[s], plan.aggPart[h] = 1, 2
                    by_canon[k + "#hi"] = h
            a.slot = by_canon[k]
            a.hi_slot = by_canon.get(k + "#hi", -1)
        self.args = args

        plan.hasWhere = 1 if where is not None else 0
        if where is not None:
            plan.where = env.compile(where)
        plan.nkeys = len(keys)
        for i, (kx, key_int) in enumerate(keys):
            plan.keys[i] = env.compile(kx)
            plan.keyInt[i] = 1 if key_int and env.is_int(plan.keys[i]) else 0
        meta = {}
        for a in aggs:
            if a.arg is not None:
                meta.setdefault(a.slot, a)
        for s in range(1, plan.naggs):
            plan.aggs[s] = env.compile(args[s])
        plan.aggInt[0] = 1
        for s in range(1, plan.naggs):
            plan.aggInt[s] = 1 if plan.ops[s] != abi.AGG_COUNT and env.is_int(plan.aggs[s]) else 0
            plan.aggNull[s] = 0
            pg = plan.aggs[s]
            if plan.ops[s] != abi.AGG_COUNT and pg.len == 1 and env.env.code[pg.start].op == abi.OP_COL:
                t = env.env.cols[env.env.code[pg.start].arg].t
                if t in (abi.T_I32N, abi.T_I64N):
                    plan.aggNull[s] = t
                    plan.aggInt[s] = 1
            a = meta.get(s) or meta.get(s - 1)
            plan.aggBits[s] = 0
            if (grouped and plan.aggInt[s] and a is not None and a.is_col and a.arg_type in ("BIGINT", "DATETIME")
                    and (plan.ops[s] in (abi.AGG_MIN, abi.AGG_MAX) or plan.aggPart[s])):
                plan.aggBits[s] = 1
        for s in range(1, plan.naggs):
            if plan.aggPart[s] == 1 and plan.aggBits[s] != plan.aggBits[s + 1]:
                plan.aggBits[s] = plan.aggBits[s + 1] = 0
        self.plan = plan


def dense_spec(plan: abi.AggPlan, ranges: list[tuple[int, int]], rows: int) -> abi.DenseSpec | None:
    """DenseSpec for GROUP BY keys with value ranges [lo, hi], or None when the engine would hash
    (src/engine_select.cpp:1172-1229)."""
    ds = abi.DenseSpec()
    G = 1
    for k, (lo, hi) in enumerate(ranges):
        span = hi - lo
        if span >= (1 << 26):
            return None
        r = span + 1
        if G > (1 << 26) // r:
            return None
        ds.kmin[k], ds.range[k], ds.stride[k] = lo, r, G
        G *= r
    off = 0
    int_only = True
    for a in range(plan.naggs):
        op, i = plan.ops[a], plan.aggInt[a]
        kind = (abi.DK_COUNT if op == abi.AGG_COUNT else (abi.DK_SUM_I if i else abi.DK_SUM_D) if op == abi.AGG_SUM
                else (abi.DK_MIN_I if i else abi.DK_MIN_D) if op == abi.AGG_MIN else (abi.DK_MAX_I if i else abi.DK_MAX_D))
        ds.kind[a] = kind
        ds.slotOff[a] = off
        nbytes = G * (4 if kind == abi.DK_COUNT else 8)
        off += min((nbytes + 7) // 8 * 8, 1 << 30)
        int_only &= kind in (abi.DK_COUNT, abi.DK_SUM_I, abi.DK_MIN_I, abi.DK_MAX_I)
    copy_bytes = off
    if G * plan.naggs <= 88:
        ds.priv, ds.G = 1, G
    elif copy_bytes <= 48 * 1024 and G < 64 and not int_only:
        return None
    elif copy_bytes <= 48 * 1024:
        ds.copies, ds.copyBytes, ds.G = min(8, (48 * 1024) // copy_bytes), copy_bytes, G
    elif G <= max(4 * rows, 1 << 16) and G * (8 + 8 * plan.nkeys + 8 * plan.naggs) <= (512 << 20):
        ds.copies, ds.G = 0, G
    else:
        return None
    plan.densePriv = 1 if ds.priv else 2
    return ds
