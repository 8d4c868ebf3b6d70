/* CPU oracle of the Warpstore hot-path operators — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement (multithreaded with std::thread) of what the engine's GPU operators
 * compute, used by the tests as the parity checker and by bench.py as the timed CPU baseline.
 * Nothing in the product library links or calls it.  Each function names the reference code whose
 * semantics it restates (paths are within the Warpstore source tree).
 *
 * Results are exact: integer SUMs as int128 (lo, hi words), COUNT / MIN / MAX as int64, DOUBLE
 * aggregates as doubles (NaN skipped); groups are identified by their exact key values.
 */
#ifndef WS_ORACLE_H
#define WS_ORACLE_H
#include "../include/ws_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ws_oracle_result ws_oracle_result;

/* Typed evaluation of one expression for one row of a batch (cols = that batch's views).
 * Returns the value as a double (NaN = NULL) and, when the expression is integer-typed, the exact
 * int64 in *ival with *is_int = 1.  *ovf is set when checked int64 arithmetic overflowed. */
/* Static type of an expression: 1 int64, 0 double, -1 malformed. */
int ws_oracle_prog_is_int(const ws_expr_env* env, ws_prog p);
/* The engine's segment encoding (Table::encodeColumn): enc (0 raw) and the bytes (when cap allows). */
int ws_oracle_encode_column_engine(const void* src, int ptype, int64_t n, uint8_t* out, int64_t cap, int64_t* bytes);
double ws_oracle_eval(const ws_expr_env* env, const ws_col_view* cols, ws_prog prog, int64_t row, int64_t* ival,
                      int* is_int, int* ovf);

/* Filter + aggregate (no keys, dense or hash GROUP BY; the semantics do not depend on the mode).
 * Batches: bn[b] rows, deleted bitmap bdel[b] (may be null), views bcols[b*ncols + c]. */
int ws_oracle_aggregate(const ws_expr_env* env, const ws_agg_plan* plan, int nb, const int64_t* bn,
                        const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int nthreads,
                        ws_oracle_result** out);
/* COUNT(DISTINCT x) next to the plan's aggregates (src/engine_select.cpp:1397-1492): one extra slot
 * per group counting the distinct non-NULL values of `distinct`. */
int ws_oracle_aggregate_distinct(const ws_expr_env* env, const ws_agg_plan* plan, ws_prog distinct, int distinct_int,
                                 int nb, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                                 int ncols, int nthreads, ws_oracle_result** out);

/* Groups sorted by their key words (int64 bits, lexicographic, signed). */
int64_t ws_oracle_ngroups(const ws_oracle_result* r);
int ws_oracle_nkeys(const ws_oracle_result* r);
int ws_oracle_naggs(const ws_oracle_result* r);
int ws_oracle_overflow(const ws_oracle_result* r);
/* keys[g * nk + k]: keyInt keys as int64, other keys as the bits of the double (+0.0 for -0.0) */
void ws_oracle_keys(const ws_oracle_result* r, int64_t* keys);
/* words[(g * na + a) * 2 + {0,1}]: int SUM (lo, hi) of the int128; COUNT / int MIN / MAX (v, 0);
 * double slots (bits, 0). */
void ws_oracle_words(const ws_oracle_result* r, int64_t* words);
void ws_oracle_free(ws_oracle_result* r);

/* Row selection: ascending global indices of rows passing `where` and not deleted
 * (src/gpu.cu:694-755).  Returns the count; idx may be null to count only; per_batch[nb]. */
int64_t ws_oracle_select(const ws_expr_env* env, int has_where, ws_prog where, int nb, const int64_t* bn,
                         const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int nthreads,
                         int32_t* idx, int64_t* per_batch);

/* Inner equi-join pairs (src/gpu.cu:1093-1193): every (build row, probe row) with equal non-NULL keys,
 * sorted by (probe, build).  Returns the count; pass null outputs to count only. */
int64_t ws_oracle_hash_join(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int nthreads,
                            int32_t* out_build, int32_t* out_probe);

/* Gather (src/gpu.cu:757-800): dst[j] = row idx[j] of the concatenated batches, decoded to ptype. */
void ws_oracle_gather_multi(const ws_col_view* src, const int64_t* boff, int nb, int ptype, int esize,
                            const int32_t* idx, int64_t m, void* dst);

/* Outer join (src/gpu.cu:1197-1293): the inner pairs, (-1, probe row) for each unmatched probe row, and
 * with full (build row, -1) for each build row that matched nothing.  Returns the count. */
int64_t ws_oracle_hash_join_outer(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int full,
                                  int32_t* out_build, int32_t* out_probe);
/* Stable multi-key sort permutation (src/gpu.cu:1323-1361): NULL as -inf, -0 as 0, desc[k] inverts. */
void ws_oracle_sort_perm(const double* const* keys, const int* desc, int nkeys, int64_t m, int32_t* perm);
/* Evaluation at rows (src/gpu.cu:862-888, :1011-1019): doubles, or int64 when as_int (exact integer
 * programs, a single integer column as stored, else the double rounded; NULL = the BIGINT sentinel). */
void ws_oracle_eval_at(const ws_expr_env* env, const ws_col_view* cols, ws_prog prog, const int32_t* idx, int64_t m,
                       int as_int, void* out, int* ovf);

#ifdef __cplusplus
}
#endif
#endif
