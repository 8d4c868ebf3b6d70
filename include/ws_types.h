/* Plain data types of the segment / expression / aggregation ABI.
 *
 * Every struct here is byte-for-byte the layout the Warpstore engine hands to its GPU operators
 * (reference: src/devtypes.h:64-102 Instr/ColView, :168-194 ExprEnv, :503-547 AggPlan/DenseSpec/
 * BatchSet).  The engine builds these values with its own bytecode compiler and passes them to the
 * operator entry points declared in ws_b200.h, so the layout is an interface that must not drift:
 * ws_abi_check() in the library and the static asserts below pin sizes and offsets.
 *
 * The header is plain C (usable from C, C++, nvcc and NVRTC-compiled query kernels); it includes
 * no host headers when compiled by NVRTC.
 */
#ifndef WS_TYPES_H
#define WS_TYPES_H

#if defined(__CUDACC_RTC__)
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits of one compiled expression set (src/devtypes.h:163-173) */
#define WS_MAX_STACK 16
#define WS_MAX_COLS 128
#define WS_MAX_CODE 320
#define WS_MAX_CONSTS 96
#define WS_MAX_SETS 16
#define WS_MAX_KEYS 8
#define WS_MAX_AGGS 64
/* plans the on-device bytecode interpreter accepts; larger plans must be compiled */
#define WS_INTERP_KEYS 4
#define WS_INTERP_AGGS 16
/* encoded segment columns start with a 16-byte header (int64 base, then a double 10^s) */
#define WS_ENC_HEADER 16

/* NULL sentinels of integer storage; doubles hold NaN (src/devtypes.h:27-28) */
#define WS_NULL_I32 ((int32_t)0x80000000)
#define WS_NULL_I64 ((int64_t)0x8000000000000000ull)

/* ---- expression bytecode: a stack program per expression (src/devtypes.h:64-83).
 * The numeric values are part of the engine's bytecode and must stay as they are. */
enum ws_op {
  WS_OP_COL = 0,   /* push column[arg][row] */
  WS_OP_CONST,     /* push consts[arg] (isInt: the double slot holds the int64 bit pattern) */
  WS_OP_ADD, WS_OP_SUB, WS_OP_MUL, WS_OP_DIV, WS_OP_MOD, WS_OP_NEG,
  WS_OP_EQ, WS_OP_NE, WS_OP_LT, WS_OP_LE, WS_OP_GT, WS_OP_GE,
  WS_OP_AND, WS_OP_OR, WS_OP_NOT,
  WS_OP_INSET,     /* dictionary code -> bit of sets[arg] */
  WS_OP_SELECT,    /* cond, then, else -> CASE WHEN */
  WS_OP_YEAR,      /* days since 1970-01-01 -> year */
  WS_OP_ISNULL,
  WS_OP_COALESCE,
  WS_OP_NULLIF,
  WS_OP_CALL1,     /* scalar function fn[arg](x), ids in ws_fn */
  WS_OP_CALL2,
  WS_OP_DICTMAP,   /* dictionary code -> maps[arg][code] */
  WS_OP_INSORTED,  /* x IN sorted maps[arg] */
  WS_OP_VDOT,      /* dot(float vector column[arg&255], maps[arg>>8]) */
  WS_OP_VEUC,      /* euclidean distance, same operands */
  WS_OP_COLRAW     /* raw stored integer of column[arg] (DECIMAL sums) */
};

/* scalar function ids (src/devtypes.h:310-322) */
enum ws_fn {
  WS_FN_ABS = 0, WS_FN_CEIL, WS_FN_FLOOR, WS_FN_ROUND, WS_FN_SQRT, WS_FN_EXP, WS_FN_LN, WS_FN_LOG10, WS_FN_LOG2,
  WS_FN_SIN, WS_FN_COS, WS_FN_TAN, WS_FN_SIGN, WS_FN_MONTH, WS_FN_DAY, WS_FN_DAYOFWEEK, WS_FN_DAYOFYEAR,
  WS_FN_QUARTER, WS_FN_WEEKDAY, WS_FN_LAST_DAY, WS_FN_DT_DATE, WS_FN_DT_HOUR, WS_FN_DT_MINUTE, WS_FN_DT_SECOND,
  WS_FN_DATE_TO_DT, WS_FN_DT_UNIX, WS_FN_UNIX_DT, WS_FN_DT_YEAR, WS_FN_DT_MONTH, WS_FN_DT_DAY, WS_FN_ASIN,
  WS_FN_ACOS, WS_FN_ATAN, WS_FN_DEGREES, WS_FN_RADIANS, WS_FN_WEEK, WS_FN_TO_DAYS, WS_FN_FROM_DAYS,
  WS_FN_DT_MICRO, WS_FN_YEARWEEK,
  WS_FN_ROUND2 = 100, WS_FN_POW, WS_FN_ATAN2, WS_FN_LEAST, WS_FN_GREATEST, WS_FN_TRUNCATE2, WS_FN_ADD_MONTHS,
  WS_FN_DT_ADD_MONTHS, WS_FN_LOG_B, WS_FN_IDIV, WS_FN_DATE_TRUNC_MONTH, WS_FN_DT_DIFF_UNIT
};

typedef struct ws_instr {
  uint8_t op;
  uint8_t isInt;
  uint16_t arg;
} ws_instr;

/* Column view of one column of one batch (segment / write buffer / joined relation).
 * t: 0 I32, 1 I64, 2 F64 (NULL = NaN), 3 I32 with NULLs, 4 I64 with NULLs, 5 float32 vectors,
 *    6 DECIMAL (int64 scaled by 10^scale).
 * enc: 0 raw; 1/2/3 uint8/uint16/uint32 offsets from the int64 base in the header (all-ones code =
 *    NULL); 4 F64 dictionary (256 doubles after the header, then uint8 codes); 5/6 decimal-valued
 *    F64 as uint16/uint32 offsets from the base, divided by the header's double 10^s (the engine's
 *    formats); 7 bit-packed and 8 run-length integer columns (this library's formats, ws_dev.cuh).
 * off: first row of a range scan (encoded columns; raw pointers are offset by the caller). */
typedef struct ws_col_view {
  const void* p;
  uint8_t t;
  uint8_t scale;
  uint8_t enc;
  int32_t off;
} ws_col_view;

typedef struct ws_prog {
  int16_t start;
  int16_t len;
} ws_prog;

/* Everything a kernel needs to evaluate one query's expressions. */
typedef struct ws_expr_env {
  ws_instr code[WS_MAX_CODE];
  double consts[WS_MAX_CONSTS];
  const uint32_t* sets[WS_MAX_SETS];
  int32_t setSize[WS_MAX_SETS];
  const double* maps[WS_MAX_SETS];
  int32_t mapSize[WS_MAX_SETS];
  ws_col_view cols[WS_MAX_COLS];
  int* ovf; /* device flag: checked BIGINT arithmetic overflowed */
} ws_expr_env;

enum ws_agg_op { WS_AGG_SUM = 0, WS_AGG_COUNT = 1, WS_AGG_MIN = 2, WS_AGG_MAX = 3 };

/* Aggregation plan (src/devtypes.h:503-520).  Slot 0 is the hidden COUNT(*).
 * aggInt: integer-valued argument (exact accumulation).  aggBits: with GROUP BY, the slot's result
 * is exact int64 bits in the double; aggPart 1/2: the low / high 32-bit halves of a BIGINT SUM.
 * aggNull: 3 / 4 = the argument is a nullable I32 / I64 column read raw, NULLs skipped. */
typedef struct ws_agg_plan {
  uint8_t hasWhere;
  ws_prog where;
  int32_t nkeys;
  ws_prog keys[WS_MAX_KEYS];
  int32_t naggs;
  ws_prog aggs[WS_MAX_AGGS];
  uint8_t ops[WS_MAX_AGGS];
  uint8_t aggInt[WS_MAX_AGGS];
  uint8_t aggBits[WS_MAX_AGGS];
  uint8_t aggPart[WS_MAX_AGGS];
  uint8_t aggNull[WS_MAX_AGGS];
  uint8_t densePriv;
  uint8_t keyInt[WS_MAX_KEYS];
  const ws_expr_env* genv;
} ws_agg_plan;

enum ws_dense_kind { WS_DK_COUNT = 0, WS_DK_SUM_I, WS_DK_SUM_D, WS_DK_MIN_I, WS_DK_MAX_I, WS_DK_MIN_D, WS_DK_MAX_D };

/* Dense GROUP BY over small known key ranges: group = sum((key_k - kmin_k) * stride_k). */
typedef struct ws_dense_spec {
  int64_t G;
  int32_t copies;
  int32_t copyBytes;
  int32_t priv;
  int64_t kmin[WS_MAX_KEYS];
  int64_t range[WS_MAX_KEYS];
  int64_t stride[WS_MAX_KEYS];
  int32_t slotOff[WS_MAX_AGGS];
  uint8_t kind[WS_MAX_AGGS];
} ws_dense_spec;

/* physical column types of gathers (src/common.h:24) */
enum ws_ptype { WS_PT_I32 = 0, WS_PT_I64 = 1, WS_PT_F64 = 2, WS_PT_VEC = 5 };
/* ws_col_view.t values */
enum ws_view_type { WS_T_I32 = 0, WS_T_I64 = 1, WS_T_F64 = 2, WS_T_I32N = 3, WS_T_I64N = 4, WS_T_VEC = 5, WS_T_DEC = 6 };
/* ws_col_view.enc values of this library's integer formats */
enum ws_enc { WS_ENC_BITPACK = 7, WS_ENC_RLE = 8 };

/* operator kinds a plan is compiled for (src/jit.h:14) */
enum ws_jit_fn { WS_JF_NOKEYS = 0, WS_JF_GROUPED = 1, WS_JF_DENSE = 2, WS_JF_FLAG = 3, WS_JF_FLAGM = 4 };
enum ws_jit_mode { WS_JIT_OFF = 0, WS_JIT_ON = 1, WS_JIT_SYNC = 2 };

#ifdef __cplusplus
}
#endif

#if defined(__cplusplus) && !defined(__CUDACC_RTC__)
static_assert(sizeof(ws_instr) == 4, "Instr layout");
static_assert(sizeof(ws_col_view) == 16, "ColView layout");
static_assert(offsetof(ws_col_view, off) == 12, "ColView layout");
static_assert(offsetof(ws_expr_env, consts) == 1280, "ExprEnv layout");
static_assert(offsetof(ws_expr_env, cols) == 2432, "ExprEnv layout");
static_assert(sizeof(ws_expr_env) == 4488, "ExprEnv layout");
static_assert(offsetof(ws_agg_plan, nkeys) == 8, "AggPlan layout");
static_assert(offsetof(ws_agg_plan, naggs) == 44, "AggPlan layout");
static_assert(offsetof(ws_agg_plan, ops) == 304, "AggPlan layout");
static_assert(offsetof(ws_agg_plan, densePriv) == 624, "AggPlan layout");
static_assert(offsetof(ws_agg_plan, genv) == 640, "AggPlan layout");
static_assert(sizeof(ws_agg_plan) == 648, "AggPlan layout");
static_assert(offsetof(ws_dense_spec, kmin) == 24, "DenseSpec layout");
static_assert(offsetof(ws_dense_spec, kind) == 472, "DenseSpec layout");
static_assert(sizeof(ws_dense_spec) == 536, "DenseSpec layout");
#endif

#endif /* WS_TYPES_H */
