/* libwarpstore_b200 — C ABI of the B200 query-execution core.
 *
 * These entry points replace the GPU operator layer of the Warpstore engine: src/gpu.h (allocation,
 * aggregation, selection, gathers, joins) and src/jit.h (per-query compiled plans and the plan cache).
 * Each declaration names the reference interface it stands in for.  The C++ engine keeps calling the
 * same C++ signatures through the header-only shim ws_gpu.hpp, which forwards here.
 *
 * Conventions
 *  - Every function returns WS_OK (0) or an error code; the message of the calling thread's last
 *    error is ws_last_error().  Codes are the engine's SQL error numbers: WS_ERR_OOM (1041) means
 *    "GPU out of memory" (the engine retries the query alone), WS_ERR_PLAN (1235) a plan the
 *    interpreter cannot run, WS_ERR_INTERNAL (1105) everything else.
 *  - Device pointers are plain CUDA device addresses.  Work is issued on the calling thread's stream
 *    (ws_set_stream; default: the per-thread default stream, as the engine is built with
 *    --default-stream per-thread).  Functions that return a count synchronize that stream.
 *  - Buffers returned through T** are stream-ordered pool allocations: release them with ws_tmp_free.
 *  - All entry points are re-entrant across threads.
 */
#ifndef WS_B200_H
#define WS_B200_H
#include "ws_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WS_OK 0
#define WS_ERR_OOM 1041
#define WS_ERR_INTERNAL 1105
#define WS_ERR_PLAN 1235
#define WS_ERR_SIZE 1206     /* an output buffer is too small: the needed size is returned */
#define WS_ERR_ARG 1210      /* invalid argument */
#define WS_ERR_RANGE 1264    /* a dense GROUP BY key outside its declared range */

/* ---- errors */
const char* ws_last_error(void);
int ws_last_error_code(void);

/* ---- device runtime (src/gpu.h:12-56: gpuInit, gpuSmCount, gpuArch, gpuDescribe, devAlloc/devFree,
 *      tmpAlloc/tmpFree, h2d/d2h/d2d, gpuSync, gpuTrimPool) */
int ws_gpu_init(void);
int ws_gpu_sm_count(void);
int ws_gpu_arch(void);
int ws_gpu_describe(char* buf, size_t size);
int ws_set_stream(void* stream); /* cudaStream_t for this thread; NULL restores the default */
void* ws_get_stream(void);
int ws_dev_alloc(size_t bytes, void** out);
int ws_dev_free(void* p);
int ws_tmp_alloc(size_t bytes, void** out);
int ws_tmp_free(void* p);
int ws_h2d(void* dst, const void* src, size_t bytes);
int ws_d2h(void* dst, const void* src, size_t bytes);
int ws_d2d(void* dst, const void* src, size_t bytes);
int ws_gpu_sync(void);
int ws_gpu_trim_pool(void);
/* Pinned host memory that kernels can write (cudaHostAlloc, mapped): the destination of
 * ws_agg_fetch_async.  No counterpart in the reference, whose pinned staging is internal. */
int ws_host_alloc(size_t bytes, void** out);
int ws_host_free(void* p);

/* ---- tiered column storage (src/gpu.h:19-47: gpuSetVramLimit, gpuVramUsed, gpuVramFill, placeColumn,
 *      releaseColumn, vramAcquire, vramRelease, hostMap, hostUnmap, gpuVramLimit, gpuVramFree).
 * Segment columns live in device memory while the library's VRAM budget (ws_set_vram_limit; default
 * none) has room, else their host bytes are pinned and mapped and kernels read them over PCIe.  Device
 * copies made here are counted against the budget until released. */
int ws_set_vram_limit(int64_t bytes);   /* INT64_MAX: no limit */
int64_t ws_vram_used(void);             /* bytes of device copies made by ws_place_column / ws_vram_acquire /
                                           ws_patch_column / ws_update_column and not yet released */
int64_t ws_vram_limit(void);
int64_t ws_vram_free(void);             /* free device memory (cudaMemGetInfo), 0 without a device */
double ws_vram_fill(void);              /* used / limit, or the device's used fraction without a limit */
/* placeColumn: *out = a device copy of host[0, bytes) (*mapped = 0) when the budget has room and
 * host_only is 0, else host is pinned + mapped and *out its device address (*mapped = 1). */
int ws_place_column(void* host, size_t bytes, int host_only, void** out, int* mapped);
int ws_release_column(void* dev, void* host, size_t bytes, int mapped);
/* vramAcquire: a device copy of host bytes, or *out = NULL when it does not fit (no error). */
int ws_vram_acquire(const void* host, size_t bytes, void** out);
int ws_vram_release(void* dev, size_t bytes);
/* hostMap: host bytes pinned + mapped, *out = their device address (NULL when registering fails). */
int ws_host_map(void* host, size_t bytes, void** out);
int ws_host_unmap(void* host);

/* ---- column-level UPDATE (src/gpu.h:24-41: gpuPatchColumn, gpuUpdateColumn).  Both return a new
 * device copy of the column (counted against the VRAM budget; release with ws_vram_release), or
 * *out = NULL when it does not fit.  rows (and vals) are host arrays of m entries. */
/* gpuPatchColumn: the column (bytes, width 4 or 8) with rows[i] set to the width-byte value vals[i]. */
int ws_patch_column(const void* old_dev, size_t bytes, int width, const int32_t* rows, const void* vals, int64_t m,
                    void** out);
/* gpuUpdateColumn (GpuUpdate, field for field): kind 0 sets rows[i] to i0 / d0, 1 to src[rows[i]],
 * 2 to src[rows[i]] + add (integers, checked) / + add_d (doubles).  Integers must stay in [lo, hi]; NULLs
 * (nul / NaN) stay NULL unless not_null (then bad).  Out: bad (nothing returned), saw_null, and mn / mx of
 * the new non-NULL values (+inf / -inf when none). */
typedef struct ws_update {
  int32_t kind;
  int64_t i0, add, nul, lo, hi;
  double d0, add_d;
  uint8_t not_null;
  uint8_t bad, saw_null;
  double mn, mx;
} ws_update;
int ws_update_column(const void* old_dev, const void* src, int64_t n, int w, int f64, const int32_t* rows, int64_t m,
                     ws_update* u, void** out);

/* ---- aggregation (src/gpu.h:84-130, class GpuAggregator).
 * Batches (segments, write buffers or a joined relation) are collected with ws_agg_add_batch and
 * aggregated by ws_agg_run in one pass.  Without GROUP BY there is one result row; with a dense spec
 * (G > 0) groups index arrays directly; otherwise an open-addressing hash table of `capacity` rows
 * (rounded up to a power of two) is used, and ws_agg_overflowed reports when it filled up (the
 * caller retries bigger, as the engine does). */
typedef struct ws_aggregator ws_aggregator;
typedef struct ws_jit_program ws_jit_program;
int ws_agg_create(const ws_agg_plan* plan, int64_t capacity, const ws_dense_spec* dense, ws_aggregator** out);
void ws_agg_destroy(ws_aggregator* agg);
int ws_agg_add_batch(ws_aggregator* agg, const ws_expr_env* env, int ncols, int64_t n, const uint32_t* del);
/* Many batches in one call (batch b: bn[b] rows, deleted bitmap bdel[b], views bcols[b * ncols ..]); the
 * same as ws_agg_add_batch per batch with env.cols set to that batch's views. */
int ws_agg_add_batches(ws_aggregator* agg, int ncols, int nb, const int64_t* bn, const uint32_t* const* bdel,
                       const ws_col_view* bcols);
int ws_agg_run(ws_aggregator* agg, const ws_expr_env* env, const ws_jit_program* jit);
int ws_agg_run_window(ws_aggregator* agg, const ws_expr_env* env, const ws_jit_program* jit);
/* Several aggregations in ONE kernel launch (no counterpart in the reference, which launches each
 * query on its own): aggs[i] over its batches with envs[i]'s constants, all of one scan kind (no GROUP
 * BY, dense private rows, or hash GROUP BY) and one compiled plan `jit` (null: all interpreted, which
 * lets queries of different expressions share the launch).  The SMs' resident CTAs are shared out by
 * the queries' tiles; each query's results are then read as after ws_agg_run.  Aggregators without
 * batches are skipped.  WS_ERR_ARG when the queries need different kernels. */
int ws_agg_run_many(ws_aggregator* const* aggs, const ws_expr_env* const* envs, const ws_jit_program* jit, int n);
int ws_agg_batches(const ws_aggregator* agg);
int ws_agg_windows(const ws_aggregator* agg);
int64_t ws_agg_rows_in(const ws_aggregator* agg);
int ws_agg_is_dense(const ws_aggregator* agg);
int64_t ws_agg_capacity(const ws_aggregator* agg);
int ws_agg_overflowed(ws_aggregator* agg, int* out);
int ws_agg_group_count(ws_aggregator* agg, int64_t* out);
/* Groups in host memory (GpuAggregator::fetch): keys[g * nkeys + k], accs[g * naggs + a] in the engine's
 * format (int64 bits for integer keys and aggBits slots; a split BIGINT SUM as its 2^32-weighted high
 * and low parts; doubles otherwise).  exact (optional) receives [g][naggs][2] int64 words: (lo, hi) of
 * the exact int128 integer SUM, (value, 0) for COUNT / integer MIN / MAX, (bits, 0) for doubles.
 * max_groups < groups: WS_ERR_SIZE with *ngroups set. */
int ws_agg_fetch(ws_aggregator* agg, int64_t max_groups, double* keys, double* accs, int64_t* exact, int64_t* ngroups);
/* The same groups without a host round trip (no counterpart in the reference; the serving loop's
 * form): queues compaction and a kernel that writes groups [first_group, first_group + max_groups) (in
 * ws_agg_fetch's order) as keys [.][nkeys] and exact [.][naggs][2] (the formats above) straight into
 * host memory, and *status, then returns.  keys, exact and status must be pinned host memory
 * (ws_host_alloc, or registered with CUDA); they are valid once the calling thread's stream has been
 * synchronised (ws_gpu_sync).  status->groups: all groups of the run (a caller with a smaller buffer
 * fetches the rest range by range; the compaction is done once per run); status->overflow: the hash
 * table filled up (ws_agg_overflowed; nothing written, rerun bigger); status->error: WS_ERR_RANGE /
 * WS_ERR_INTERNAL where ws_agg_fetch would raise them (nothing written). */
typedef struct ws_fetch_status {
  int64_t groups;
  int32_t overflow;
  int32_t error;
} ws_fetch_status;
int ws_agg_fetch_async(ws_aggregator* agg, int64_t first_group, int64_t max_groups, double* keys, int64_t* exact,
                       ws_fetch_status* status);
/* ---- prepared queries (no counterpart in the reference, which launches every query afresh).  The
 * aggregation of `plan` over the batches, built once: result rows, batch descriptor, and one CUDA graph
 * of the whole query (rows reset, the scan, compaction, the groups and a ws_fetch_status written into
 * pinned host memory owned by the executor, up to max_groups groups).  ws_exec_run queues the graph on
 * the calling thread's stream with env's constants, sets and maps (its expressions must be those of
 * the env given at creation: WS_ERR_ARG otherwise); after the stream is synchronised ws_exec_results
 * gives the groups (ws_agg_fetch's formats), valid until the next run.  status->overflow: the hash
 * table filled up (create a bigger one); status->groups > max_groups: only max_groups were written.
 * Needs a compiled plan covering the batches (WS_ERR_PLAN otherwise).  One run at a time per executor;
 * destroy it from the thread whose stream ran it. */
typedef struct ws_executor ws_executor;
int ws_exec_create(const ws_agg_plan* plan, int64_t capacity, const ws_dense_spec* dense, const ws_expr_env* env,
                   int ncols, int nb, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                   const ws_jit_program* jit, int64_t max_groups, ws_executor** out);
int ws_exec_run(ws_executor* ex, const ws_expr_env* env);
int ws_exec_results(ws_executor* ex, const double** keys, const int64_t** exact, const ws_fetch_status** status);
void ws_exec_destroy(ws_executor* ex);
/* Several prepared queries run as one (no counterpart in the reference): one CUDA graph that resets
 * every query's result rows, runs ONE multi-query scan over all of them (as ws_agg_run_many) and then
 * delivers each query's groups and status into its own executor's pinned memory (read them with
 * ws_exec_results).  The executors must share one compiled plan (`jit`) and a scan kind with a
 * multi-query form (hash, dense private rows, no keys; direct loads): WS_ERR_ARG otherwise.
 * ws_exec_group_run takes one env per executor, in the order given at creation, each with the
 * expressions of its executor's; it first waits until the group's previous run has read its
 * constants.  While a group runs, its executors must not run on their own; destroy the group before
 * its executors, from the thread whose stream ran it. */
typedef struct ws_exec_group ws_exec_group;
int ws_exec_group_create(ws_executor* const* exs, int n, const ws_jit_program* jit, ws_exec_group** out);
int ws_exec_group_run(ws_exec_group* g, const ws_expr_env* const* envs);
void ws_exec_group_destroy(ws_exec_group* g);

/* Without GROUP BY: which slots hold exact int64 bits (GpuAggregator::sumBitsSlots) and the high 64 bits
 * of the exact integer sums (GpuAggregator::sumHigh; valid after ws_agg_fetch). */
int ws_agg_sum_bits_slots(const ws_aggregator* agg, uint8_t* out);
int ws_agg_sum_high(const ws_aggregator* agg, int64_t* out);
/* Groups left in device memory, column-major (GpuAggregator::compact): keys[k * g + i], accs[a * g + i]. */
int ws_agg_compact(ws_aggregator* agg, double** keys, double** accs, int64_t* ngroups);

/* ---- aggregation without any allocation.  No counterpart in the reference: an addition for callers
 * that may not allocate device memory (code running where the allocator is off limits, or under a
 * memory budget owned by someone else).  Filter + aggregates without GROUP BY over the batches, like
 * ws_agg_create / add_batch / run / fetch with nkeys = 0, but all scratch (batch descriptor, per-CTA
 * partial rows, result row, control words) lives in one fixed array of WS_NOALLOC_SCRATCH_BYTES inside
 * this library, held on every GPU that loads it until the process exits.  The caller passes the plan,
 * the column views and `exact`, a host array of plan->naggs * 2 words that receives the result in the
 * format of ws_agg_fetch's `exact`.  jit: a compiled WS_JF_NOKEYS plan, or null for the interpreter.
 * Limits: the batch descriptor (about nb * (ncols * 16 + 32) bytes, plus 9 KiB interpreted) must fit
 * 1 MiB, else WS_ERR_SIZE.  Every call shares the array and reinitialises it; calls that overlap on
 * the GPU race, so serialise them.  The first call on each device looks up the array's address (do
 * it before any stream capture) and keeps it for the process: after a cudaDeviceReset of that device
 * the address no longer holds, so the entry must not be called again. */
#define WS_NOALLOC_SCRATCH_BYTES (4u << 20)
int ws_agg_nokeys_noalloc(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, const ws_jit_program* jit,
                          int nb, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                          int64_t* exact);

/* ---- selection and gathers (src/gpu.h:132-143, :170-172) */
int ws_select(const ws_expr_env* env, int has_where, ws_prog where, int64_t n, const uint32_t* del, int32_t* out_idx,
              const ws_jit_program* jit, int64_t* count);
int ws_select_multi(const ws_expr_env* env, int has_where, ws_prog where, int nb, const int64_t* bn,
                    const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int32_t** out_idx,
                    int64_t* per_batch, const ws_jit_program* jit, int64_t* count);
int ws_gather_multi(const ws_col_view* src, const int64_t* boff, int nb, int ptype, int esize, const int32_t* idx,
                    int64_t m, void* dst);
int ws_gather(const void* src, int ptype, const int32_t* idx, int64_t m, void* dst);

/* ---- joins (src/gpu.h:178-186: gpuHashJoin, gpuHashJoinParts).  Output pairs (build row, probe row)
 * are grouped by probe partition; out_off (optional, npparts + 1) receives each partition's first pair. */
int ws_hash_join_parts(ws_col_view build_key, const int64_t* boff, int nbparts, ws_col_view probe_key,
                       const int64_t* poff, int npparts, int32_t** out_build, int32_t** out_probe, int64_t* out_off,
                       int64_t* m);
int ws_hash_join(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int32_t** out_build,
                 int32_t** out_probe, int64_t* m);
/* ws_hash_join with the pair buffers' first capacity chosen by the caller (a predicted pair count, for
 * instance) instead of the probe rows: a join that emits more pairs runs a second time with exact sizes,
 * so only the memory held and *attempts (1 or 2) depend on it, never the pairs.  A first capacity below
 * 0.35 x the probe rows also says that most probe rows find no match: a hash-table join of 2^20 build
 * keys or more then builds a key filter (16 bits per key, held by L2) that spares those rows their
 * table access. */
int ws_hash_join_sized(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int64_t first_capacity,
                       int32_t** out_build, int32_t** out_probe, int64_t* m, int* attempts);
/* gpuHashJoinOuter (src/gpu.h:187-188): every probe row appears, with build row -1 when it matched
 * nothing (NULL keys never match); full != 0 also appends each build row that matched nothing, with
 * probe row -1.  Pairs are freed with ws_tmp_free. */
int ws_hash_join_outer(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int full,
                       int32_t** out_build, int32_t** out_probe, int64_t* m);
/* gpuCrossJoin (src/gpu.h:189): out_a[i] = i / nb, out_b[i] = i % nb; more than 200,000,000 pairs is
 * an error (WS_ERR_INTERNAL, as the engine's). */
int ws_cross_join(int64_t na, int64_t nb, int32_t** out_a, int32_t** out_b, int64_t* m);
/* gpuKeyBitmap (src/gpu.h:174): bits[] (nbits bits, cleared first) gets bit (key - lo) of every
 * non-NULL key in [lo, lo + nbits). */
int ws_key_bitmap(ws_col_view key, int64_t n, int64_t lo, int64_t nbits, uint32_t* bits);
/* gpuSetBits (src/gpu.h:176): sets bit idx[j] for every j (deleted-row bitmaps). */
int ws_set_bits(uint32_t* bits, const int32_t* idx, int64_t m);

/* ---- codes, gathers with NULLs, evaluation at rows (src/gpu.h:145-172, :190-195) */
/* gpuRemapCodes: out[i] = map[in[i]]; NULL stays NULL, codes outside [0, map_n) give -2. */
int ws_remap_codes(const int32_t* in, int64_t n, const int32_t* map, int64_t map_n, int32_t* out);
/* gpuBitsToDouble: dst[j] = (double) of the int64 stored bit for bit in src[j]. */
int ws_bits_to_double(const double* src, int64_t n, double* dst);
/* gpuGatherNull: like ws_gather, index -1 writes the type's NULL (ptype WS_PT_I32 / I64 / F64). */
int ws_gather_null(const void* src, int ptype, const int32_t* idx, int64_t m, void* dst);
/* gpuGatherBytes: elements of esize bytes (a multiple of 4); index -1 gives a NULL element (every
 * 32-bit word a NaN float when nulls != 0, else zeros). */
int ws_gather_bytes(const void* src, int esize, const int32_t* idx, int64_t m, void* dst, int nulls);
/* gpuGatherEnc: raw values of an encoded segment column (view.enc != 0) at idx, as ptype. */
int ws_gather_enc(ws_col_view view, int ptype, const int32_t* idx, int64_t m, void* dst);
/* gpuEvalAt: out[j] = prog at row idx[j] (row j when idx is null), as a double (NULL = NaN). */
int ws_eval_at(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, double* out);
/* gpuEvalAtInt: the same as int64 (NULL = the BIGINT sentinel): a single integer column exactly,
 * integer programs exactly (checked arithmetic), other programs rounded from their double value. */
int ws_eval_at_int(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, int64_t* out);

/* ---- segment encoding (the flush path, src/storage.cu:1138-1192) */
/* Encodes an integer column of n rows (t: WS_T_I32 / I64 / I32N / I64N; device memory) as one
 * segment column in a format the scan kernels decode: enc WS_ENC_BITPACK (7), WS_ENC_RLE (8), or 0 to
 * choose the smaller of the two.  *out (ws_tmp_free) receives *bytes bytes; *enc_used the format.
 * Bit-packing a range wider than 32 bits is WS_ERR_RANGE.  No counterpart in the reference, whose
 * encoder runs on the host and writes the formats 1-6. */
int ws_encode_column(const void* src, int t, int64_t n, int enc, void** out, int64_t* bytes, int* enc_used);

/* Table::encodeColumn (src/storage.cu:1138-1192) on the device: a segment column of n values (ptype
 * WS_PT_I32 / I64 / F64, device memory) in the engine's own formats, by the engine's rule: integers
 * whose value range fits as uint8 / uint16 (/ uint32 for BIGINT) offsets from the minimum (enc 1 / 2 /
 * 3); doubles with at most 255 distinct bit patterns as a dictionary (enc 4, entries in order of first
 * occurrence); other doubles that are exact decimals with at most 4 digits after the point as uint16 /
 * uint32 offsets (enc 5 / 6, the first scale that holds every value decides); otherwise, and for fewer
 * than 1024 rows, *enc_used = 0 (keep the column raw, *out = NULL).  *out (ws_tmp_free) receives
 * *bytes bytes: the 16-byte header, the dictionary (enc 4), the codes and 16 pad bytes. */
int ws_encode_column_engine(const void* src, int ptype, int64_t n, void** out, int64_t* bytes, int* enc_used);

/* ---- group-count estimation for hash table sizing (no counterpart in the reference, which sizes
 * tables from dictionary sizes and segment min/max: src/engine_select.cpp:1154-1167) */
/* HyperLogLog sketch (2^p registers, p 4..12) of the GROUP BY key(s) of the rows that pass the plan's
 * filter, over the global rows k * stride of the batches (stride = max(1, rows / sample_rows)):
 * register j = max over sampled hashes h = mix64(key bits) with top p bits j of (leading zeros of
 * h << p) + 1.  regs_out: host array of 2^p words; *sampled / *passing: sampled rows (not deleted) and
 * those that pass the filter.  A plan without keys only counts (the registers stay 0): the sampled
 * selectivity of its filter. */
int ws_hll_sketch(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int nb, const int64_t* bn,
                  const uint32_t* const* bdel, const ws_col_view* bcols, int p, int64_t sample_rows, uint32_t* regs_out,
                  int64_t* sampled, int64_t* passing);
/* Coordinated sample of a join key column (device view of n rows; keys as the joins read them, NULLs
 * skipped): the hashes mix64(key) below tau, copied to the host array out[0, min(count, cap)) in no
 * order; *count = every qualifying key.  Two sides sampled with one tau keep exactly the keys of both
 * whose hash is below it, so the join of the samples holds every pair of those keys (the estimator's
 * join-size feature; no counterpart in the reference). */
int ws_join_key_sample(ws_col_view key, int64_t n, uint64_t tau, uint64_t* out, int64_t cap, int64_t* count);
/* y[r] of a 3-layer MLP over host feature rows x[rows][features]: relu(x W1 + b1) -> relu(. W2 + b2) ->
 * . W3 + b3, weights as BF16 bits (W1 [features][hidden], W2 [hidden][hidden], W3 [hidden]), biases and
 * accumulation FP32; features <= 64, hidden a multiple of 32 up to 128. */
int ws_mlp_infer(const float* x, int rows, int features, int hidden, const uint16_t* w1_bf16, const float* b1,
                 const uint16_t* w2_bf16, const float* b2, const uint16_t* w3_bf16, float b3, float* y);

/* ---- launch-shape autotuner (no counterpart in the reference, whose launch shapes are fixed,
 * src/gpu.cu:393-653).  Per (scan kernel, plan, size class = log2 of the scan's tiles): the CTAs per
 * SM of the persistent grid, for the hash scan the per-CTA shared table's budget, for compiled no-key
 * and private-row scans the TMA staging depth; per (log2 build keys, log2 probe rows) of a hash join
 * with one build and one probe partition and a one-pass table: its slots per build key (2, 3 or 4).
 * WS_TUNE_ON: a key seen for the first time is tuned on the query's own data (each candidate timed on
 * the calling stream from reset state; the fastest is kept and the final run uses it, so results never
 * depend on tuning); WS_TUNE_USE (default): recorded choices are used, others get the default shape;
 * WS_TUNE_OFF: default shapes.  The table is kept in memory and in the plan-cache directory
 * (ws_jit_set_cache_dir).  Only fresh aggregators (no earlier window) tune. */
#define WS_TUNE_USE 0
#define WS_TUNE_ON 1
#define WS_TUNE_OFF 2
int ws_tune_set_mode(int mode);
/* The table as text, one line per key: `key ctas_per_sm smem_kb stages join_slots_per_key microseconds`
 * (ws_tune_load also reads lines without the stages and slots fields). */
int ws_tune_table(char* buf, size_t size, size_t* needed);
int ws_tune_load(const char* text);   /* adds / replaces entries from such text */
int ws_tune_clear(void);

/* ---- request loop (no counterpart in the reference, whose connections each run their query
 * synchronously): prepared GROUP BY queries served by `slots` host threads with a CUDA stream each,
 * in arrival order, admitted while the footprints of the queries in flight fit hbm_budget.
 * Results go to the query's arrays when it has them, else (arena_bytes > 0) to the worker's own
 * buffer, where each delivery is folded into the query's digest when `checksum` is set (the buffer
 * is reused by the worker's next query, as a server's send buffer is), else they stay on the device.
 * one_sync: queries run in the one-sync form (ws_agg_fetch_async into pinned memory: the thread waits
 * once per run, or once per arena-sized range of a larger result) when their arrays (keys, exact; no
 * accs) are pinned host memory (ws_host_alloc), or into the arena (pinned); otherwise queries follow
 * the engine's sequence of ws_agg_overflowed / ws_agg_fetch (into pageable arrays or arena). */
typedef struct ws_serve_query {
  /* in */
  const ws_expr_env* env;
  int ncols;
  const ws_agg_plan* plan;
  const ws_jit_program* jit;        /* compiled plan, or null (interpreter) */
  int nb;
  const int64_t* bn;
  const uint32_t* const* bdel;
  const ws_col_view* bcols;
  int64_t cap_plain;                /* hash table capacity of the plain sizing rule */
  double key_range;                 /* product of the keys' value ranges (0: unknown) */
  double arrival_s;                 /* seconds from the start of ws_serve */
  int64_t footprint;                /* device bytes the query may hold while it runs */
  int64_t max_groups;               /* capacity of the result arrays below */
  double* keys;                     /* [max_groups][nkeys], as ws_agg_fetch (may be null) */
  double* accs;                     /* [max_groups][naggs] (may be null) */
  int64_t* exact;                   /* [max_groups][naggs][2] (may be null) */
  /* out */
  double start_s, finish_s;         /* admitted, done (seconds from the start) */
  int runs;                         /* aggregation runs (1 + overflow reruns) */
  int64_t cap_used, groups;
  uint64_t checksum;                /* with `checksum`: sum over the groups of a hash of their key bits and
                                       exact words (DOUBLE SUM slots excluded) -- order-independent */
  double fsum;                      /* with `checksum`: the sum of the DOUBLE SUM slots over the groups */
} ws_serve_query;
/* Learned sizing (est may be null for the plain rule): the estimator's group-count MLP (10 features,
 * `hidden` units, BF16 weight bits), its input normalisation, the capacity margin (2^(p90 of the log2
 * underestimates)) and the gate of its correction. */
typedef struct ws_estimator_weights {
  int hidden;
  const uint16_t* w1;
  const float* b1;
  const uint16_t* w2;
  const float* b2;
  const uint16_t* w3;
  float b3;
  const float* mean;
  const float* std;
  double margin;
  float gate;                       /* the correction applies only where |correction| > gate (log2) */
} ws_estimator_weights;
typedef struct ws_serve_options {
  int slots;                        /* worker threads (queries in flight), 1..256 */
  int64_t hbm_budget;               /* admission: device bytes of the queries in flight */
  const ws_estimator_weights* est;  /* learned sizing of large hash tables; null: the plain rule */
  int one_sync;                     /* the one-sync form (see above) */
  int64_t arena_bytes;              /* per worker, for queries without result arrays (0: none) */
  int checksum;                     /* digest every delivered group (checksum, fsum) */
  int batch;                        /* up to this many arrived queries of one plan share a launch
                                       (ws_agg_run_many) before their groups are delivered one by one;
                                       0 or 1: a launch per query */
} ws_serve_options;
int ws_serve(ws_serve_query* queries, int n, const ws_serve_options* opt, double* wall_s);

/* ---- distinct values, bitmaps and temp-table columns (src/gpu.h:150-167) */
/* gpuDistinctInts: the distinct values in [base, base + span) of an integer expression at rows idx[j]
 * (rows 0..m-1 when idx is null), ascending, NULLs skipped.  As the engine's: only programs built of
 * integer columns (t 0, 1, 3, 4), integer literals, + - * and negation (stack depth <= 16) are
 * evaluated (checked arithmetic); any other program yields no values.  out: max_out slots; fewer than
 * the count: WS_ERR_SIZE with *count set. */
int ws_distinct_ints(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, int64_t base,
                     int64_t span, int64_t* out, int64_t max_out, int64_t* count);
/* gpuBitsFromColumn: *bits (nbits bits, cleared, at least one word; free with ws_dev_free) gets bit
 * (v - base) of every non-NULL value v in [base, base + nbits) of an INT (out 0) / BIGINT (out 1) device
 * column of n values; *saw_null: any NULL. */
int ws_bits_from_column(const void* col, int out, int64_t n, int64_t base, int64_t nbits, uint32_t** bits,
                        int* saw_null);
/* gpuTempColumn (TempColSpec, field for field): one column of a temp table built from compacted GROUP BY
 * results (keys [k * g + i], accs [a * g + i] on the device).  src 0: key idx; 1: aggregate slot idx with
 * kind 0 value / div, 1 int64 bits, 2 split sum (hi * 2^32 + lo), 3 count, 4 average (sum / div / count);
 * cnt >= 0: a group whose cnt slot is 0 is NULL; mul != 1 multiplies into a double.  out 0 int32, 1 int64,
 * 2 double (NULLs: sentinels / NaN).  *col (ws_dev_free): g values; *mn / *mx: of an integer output
 * (-inf / +inf for doubles or no value). */
typedef struct ws_temp_col_spec {
  int8_t src;
  int32_t idx, hi, cnt;
  uint8_t kind, key_int, sum_bits, out;
  double div, mul;
} ws_temp_col_spec;
int ws_temp_column(const double* keys, int nk, const double* accs, int na, int64_t g, const ws_temp_col_spec* s,
                   void** col, double* mn, double* mx);

/* ---- ORDER BY (src/gpu.h:197-199) */
/* gpuSortPerm: stable permutation sorting rows 0..m-1 by keys[0] (most significant) .. keys[nkeys-1],
 * each ascending or descending (desc[k] != 0); NULL (NaN) sorts as -inf (first ascending, last
 * descending), -0 as 0.  *out_perm (m int32, ws_tmp_free) receives the row order. */
int ws_sort_perm(const double* const* keys, const int* desc, int nkeys, int64_t m, int32_t** out_perm);
/* gpuMapRank: keys[j] = rank[(int)keys[j]] (dictionary code -> lexicographic rank), NULL -> -1. */
int ws_map_rank(double* keys, const int32_t* rank, int64_t m);
/* gpuSortPermHost: the stable ascending sort permutation of a host column (ptype WS_PT_I32 / I64 / F64,
 * keys compared as doubles), into the host array perm[n] (used when flushing sorted segments). */
int ws_sort_perm_host(const void* host_col, int ptype, int64_t n, int32_t* perm);

/* ---- compiled plans (src/jit.h:33-75) */
typedef struct ws_jit_info {
  int id;
  int fn_kind;
  int state;       /* 0 compiling, 1 ready, 2 failed */
  int from_disk;
  double compile_ms;
  int64_t execs;
  double total_ms, last_ms;
  int64_t source_bytes;
} ws_jit_info;
typedef struct ws_jit_query_info {
  int compiled, hits, from_disk, background;
  double compile_ms;
} ws_jit_query_info;
int ws_jit_set_mode(int mode);          /* this thread: WS_JIT_OFF / ON / SYNC */
int ws_jit_mode(void);
int ws_jit_set_default_mode(int mode);
int ws_jit_set_cache_dir(const char* dir);  /* also holds the autotuner's table (wsb200_tune.txt) */
/* The compiled plan for `fn` over the plan's expressions (nullptr in *out: run interpreted). */
int ws_jit_get(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, const char* kind,
               const ws_jit_program** out);
int ws_prog_is_int(const ws_expr_env* env, ws_prog p);
int ws_jit_program_info(const ws_jit_program* p, ws_jit_info* info);
int ws_jit_source_of(int id, char* buf, size_t size, size_t* needed);
/* The kind (field 0: "aggregate (dense)", ...), query text (1: the query that first compiled it) or
 * generated source (2) of a cached plan (jitPlanCache / jitSourceOf, src/jit.h:61-73). */
int ws_jit_plan_text(int id, int field, char* buf, size_t size, size_t* needed);
/* Ids of the plans the calling thread's last query (ws_jit_begin_query .. ws_jit_end_query) used
 * (JitQueryInfo::ids, src/jit.h:51-56); WS_ERR_SIZE when more than max_ids, with *n set. */
int ws_jit_last_query_plans(int* ids, int max_ids, int* n);
int ws_jit_plan_cache_count(void);
int ws_jit_plan_cache_row(int i, ws_jit_info* info);
int ws_jit_clear_cache(void);
int ws_jit_begin_query(const char* sql);
int ws_jit_end_query(double query_ms, ws_jit_query_info* info);

/* Generated evaluator source of a plan (what ws_jit_get compiles; host only, no device needed). */
int ws_codegen_source(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, char* buf, size_t size,
                      size_t* needed);
/* Compiles a plan's module with NVRTC for sm_<arch_sm> without loading it (host only, no device):
 * a build check of the generated code. */
int ws_codegen_compile_check(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, int arch_sm,
                             size_t* cubin_bytes);

/* ---- introspection */
/* Layout check: out[0..] = sizeof / offsetof values of the ABI structs as this library sees them. */
int ws_abi_layout(int64_t* out, int n);
/* Kernels this library has launched since it was loaded (all threads). */
int64_t ws_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* WS_B200_H */
