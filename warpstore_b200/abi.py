"""ctypes mirror of the ABI structs in include/ws_types.h (the engine's Instr / ColView / ExprEnv /
AggPlan / DenseSpec layout, src/devtypes.h:64-547)."""
from __future__ import annotations

import ctypes as C

MAX_STACK, MAX_COLS, MAX_CODE, MAX_CONSTS, MAX_SETS, MAX_KEYS, MAX_AGGS = 16, 128, 320, 96, 16, 8, 64
INTERP_KEYS, INTERP_AGGS = 4, 16
ENC_HEADER = 16
NULL_I32 = -(1 << 31)
NULL_I64 = -(1 << 63)

# opcodes (enum ws_op)
(OP_COL, OP_CONST, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MOD, OP_NEG, OP_EQ, OP_NE, OP_LT, OP_LE, OP_GT, OP_GE,
 OP_AND, OP_OR, OP_NOT, OP_INSET, OP_SELECT, OP_YEAR, OP_ISNULL, OP_COALESCE, OP_NULLIF, OP_CALL1, OP_CALL2,
 OP_DICTMAP, OP_INSORTED, OP_VDOT, OP_VEUC, OP_COLRAW) = range(30)

# scalar function ids (enum ws_fn)
FN = {name: i for i, name in enumerate(
    "ABS CEIL FLOOR ROUND SQRT EXP LN LOG10 LOG2 SIN COS TAN SIGN MONTH DAY DAYOFWEEK DAYOFYEAR QUARTER WEEKDAY "
    "LAST_DAY DT_DATE DT_HOUR DT_MINUTE DT_SECOND DATE_TO_DT DT_UNIX UNIX_DT DT_YEAR DT_MONTH DT_DAY ASIN ACOS ATAN "
    "DEGREES RADIANS WEEK TO_DAYS FROM_DAYS DT_MICRO YEARWEEK".split())}
FN.update({name: 100 + i for i, name in enumerate(
    "ROUND2 POW ATAN2 LEAST GREATEST TRUNCATE2 ADD_MONTHS DT_ADD_MONTHS LOG_B IDIV DATE_TRUNC_MONTH DT_DIFF_UNIT".split())})

AGG_SUM, AGG_COUNT, AGG_MIN, AGG_MAX = 0, 1, 2, 3
DK_COUNT, DK_SUM_I, DK_SUM_D, DK_MIN_I, DK_MAX_I, DK_MIN_D, DK_MAX_D = range(7)
PT_I32, PT_I64, PT_F64, PT_VEC = 0, 1, 2, 5
JF_NOKEYS, JF_GROUPED, JF_DENSE, JF_FLAG, JF_FLAGM = range(5)
JIT_OFF, JIT_ON, JIT_SYNC = 0, 1, 2

# column view types (ColView.t)
T_I32, T_I64, T_F64, T_I32N, T_I64N, T_VEC, T_DEC = 0, 1, 2, 3, 4, 5, 6


class Instr(C.Structure):
    _fields_ = [("op", C.c_uint8), ("isInt", C.c_uint8), ("arg", C.c_uint16)]


class ColView(C.Structure):
    _fields_ = [("p", C.c_void_p), ("t", C.c_uint8), ("scale", C.c_uint8), ("enc", C.c_uint8), ("off", C.c_int32)]


class Prog(C.Structure):
    _fields_ = [("start", C.c_int16), ("len", C.c_int16)]


class ExprEnv(C.Structure):
    _fields_ = [("code", Instr * MAX_CODE), ("consts", C.c_double * MAX_CONSTS), ("sets", C.c_void_p * MAX_SETS),
                ("setSize", C.c_int32 * MAX_SETS), ("maps", C.c_void_p * MAX_SETS), ("mapSize", C.c_int32 * MAX_SETS),
                ("cols", ColView * MAX_COLS), ("ovf", C.c_void_p)]


class AggPlan(C.Structure):
    _fields_ = [("hasWhere", C.c_uint8), ("where", Prog), ("nkeys", C.c_int32), ("keys", Prog * MAX_KEYS),
                ("naggs", C.c_int32), ("aggs", Prog * MAX_AGGS), ("ops", C.c_uint8 * MAX_AGGS),
                ("aggInt", C.c_uint8 * MAX_AGGS), ("aggBits", C.c_uint8 * MAX_AGGS), ("aggPart", C.c_uint8 * MAX_AGGS),
                ("aggNull", C.c_uint8 * MAX_AGGS), ("densePriv", C.c_uint8), ("keyInt", C.c_uint8 * MAX_KEYS),
                ("genv", C.c_void_p)]


class DenseSpec(C.Structure):
    _fields_ = [("G", C.c_int64), ("copies", C.c_int32), ("copyBytes", C.c_int32), ("priv", C.c_int32),
                ("kmin", C.c_int64 * MAX_KEYS), ("range", C.c_int64 * MAX_KEYS), ("stride", C.c_int64 * MAX_KEYS),
                ("slotOff", C.c_int32 * MAX_AGGS), ("kind", C.c_uint8 * MAX_AGGS)]


class JitInfo(C.Structure):
    _fields_ = [("id", C.c_int), ("fn_kind", C.c_int), ("state", C.c_int), ("from_disk", C.c_int),
                ("compile_ms", C.c_double), ("execs", C.c_int64), ("total_ms", C.c_double), ("last_ms", C.c_double),
                ("source_bytes", C.c_int64)]


class JitQueryInfo(C.Structure):
    _fields_ = [("compiled", C.c_int), ("hits", C.c_int), ("from_disk", C.c_int), ("background", C.c_int),
                ("compile_ms", C.c_double)]


def layout() -> list[int]:
    """sizeof / offsetof values in the order of ws_abi_layout() (runtime side of the layout check)."""
    o = C.sizeof
    return [o(Instr), o(ColView), ColView.off.offset, o(ExprEnv), ExprEnv.consts.offset, ExprEnv.sets.offset,
            ExprEnv.setSize.offset, ExprEnv.maps.offset, ExprEnv.mapSize.offset, ExprEnv.cols.offset,
            ExprEnv.ovf.offset, o(AggPlan), AggPlan.where.offset, AggPlan.nkeys.offset, AggPlan.keys.offset,
            AggPlan.naggs.offset, AggPlan.aggs.offset, AggPlan.ops.offset, AggPlan.aggInt.offset,
            AggPlan.aggBits.offset, AggPlan.aggPart.offset, AggPlan.aggNull.offset, AggPlan.densePriv.offset,
            AggPlan.keyInt.offset, AggPlan.genv.offset, o(DenseSpec), DenseSpec.kmin.offset, DenseSpec.range.offset,
            DenseSpec.stride.offset, DenseSpec.slotOff.offset, DenseSpec.kind.offset]


class ServeQuery(C.Structure):
    """ws_serve_query (include/ws_b200.h)."""
    _fields_ = [("env", C.c_void_p), ("ncols", C.c_int), ("plan", C.c_void_p), ("jit", C.c_void_p), ("nb", C.c_int),
                ("bn", C.c_void_p), ("bdel", C.c_void_p), ("bcols", C.c_void_p), ("cap_plain", C.c_int64),
                ("key_range", C.c_double), ("arrival_s", C.c_double), ("footprint", C.c_int64),
                ("max_groups", C.c_int64), ("keys", C.c_void_p), ("accs", C.c_void_p), ("exact", C.c_void_p),
                ("start_s", C.c_double), ("finish_s", C.c_double), ("runs", C.c_int), ("cap_used", C.c_int64),
                ("groups", C.c_int64), ("checksum", C.c_uint64), ("fsum", C.c_double)]


class ServeOptions(C.Structure):
    """ws_serve_options (include/ws_b200.h)."""
    _fields_ = [("slots", C.c_int), ("hbm_budget", C.c_int64), ("est", C.c_void_p), ("one_sync", C.c_int),
                ("arena_bytes", C.c_int64), ("checksum", C.c_int), ("batch", C.c_int)]


class FetchStatus(C.Structure):
    """ws_fetch_status (include/ws_b200.h)."""
    _fields_ = [("groups", C.c_int64), ("overflow", C.c_int32), ("error", C.c_int32)]


class Update(C.Structure):
    """ws_update (include/ws_b200.h; the engine's GpuUpdate)."""
    _fields_ = [("kind", C.c_int32), ("i0", C.c_int64), ("add", C.c_int64), ("nul", C.c_int64), ("lo", C.c_int64),
                ("hi", C.c_int64), ("d0", C.c_double), ("add_d", C.c_double), ("not_null", C.c_uint8),
                ("bad", C.c_uint8), ("saw_null", C.c_uint8), ("mn", C.c_double), ("mx", C.c_double)]


class TempColSpec(C.Structure):
    """ws_temp_col_spec (include/ws_b200.h; the engine's TempColSpec)."""
    _fields_ = [("src", C.c_int8), ("idx", C.c_int32), ("hi", C.c_int32), ("cnt", C.c_int32), ("kind", C.c_uint8),
                ("key_int", C.c_uint8), ("sum_bits", C.c_uint8), ("out", C.c_uint8), ("div", C.c_double),
                ("mul", C.c_double)]


class EstimatorWeights(C.Structure):
    """ws_estimator_weights (include/ws_b200.h)."""
    _fields_ = [("hidden", C.c_int), ("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_float), ("mean", C.c_void_p), ("std", C.c_void_p),
                ("margin", C.c_double), ("gate", C.c_float)]
