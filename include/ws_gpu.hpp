// Header-only C++ shim: the Warpstore engine's GPU operator interface (src/gpu.h, src/jit.h) over the
// C ABI of libwarpstore_b200 (ws_b200.h).  An engine build that includes this header instead of
// compiling src/gpu.cu and src/jit.cu calls the same C++ signatures; every call forwards to the C ABI
// and C-ABI errors are rethrown as the engine's SqlError (define WS_GPU_THROW before including this
// header; by default a std::runtime_error carrying the code is thrown).
//
// The engine's own devtypes.h defines ColView / ExprEnv / AggPlan / DenseSpec / Prog with the same
// layout as ws_types.h (checked below); define WS_GPU_ENGINE_TYPES when it is included first.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ws_b200.h"

#ifndef WS_GPU_THROW
namespace gdb {
struct WsGpuError : std::runtime_error {
  int code;
  WsGpuError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};
}  // namespace gdb
#define WS_GPU_THROW(msg, code) throw ::gdb::WsGpuError((msg), (code))
#endif

namespace gdb {

#ifndef WS_GPU_ENGINE_TYPES
using ColView = ws_col_view;
using ExprEnv = ws_expr_env;
using AggPlan = ws_agg_plan;
using DenseSpec = ws_dense_spec;
using Prog = ws_prog;
#endif
static_assert(sizeof(ColView) == sizeof(ws_col_view) && sizeof(ExprEnv) == sizeof(ws_expr_env) &&
                  sizeof(AggPlan) == sizeof(ws_agg_plan) && sizeof(DenseSpec) == sizeof(ws_dense_spec),
              "engine ABI structs and ws_types.h differ");

inline void wsCheck(int rc) {
  if (rc != WS_OK) WS_GPU_THROW(std::string(ws_last_error()), rc);
}

// ---- device runtime (src/gpu.h:12-56)
inline void gpuInit() { wsCheck(ws_gpu_init()); }
inline int gpuSmCount() { return ws_gpu_sm_count(); }
inline int gpuArch() { return ws_gpu_arch(); }
inline std::string gpuDescribe() {
  char buf[256] = {};
  wsCheck(ws_gpu_describe(buf, sizeof buf));
  return buf;
}
inline void* devAlloc(size_t bytes) {
  void* p = nullptr;
  wsCheck(ws_dev_alloc(bytes, &p));
  return p;
}
inline void devFree(void* p) { ws_dev_free(p); }
inline void* tmpAlloc(size_t bytes) {
  void* p = nullptr;
  wsCheck(ws_tmp_alloc(bytes, &p));
  return p;
}
inline void tmpFree(void* p) { ws_tmp_free(p); }
inline void gpuTrimPool() { ws_gpu_trim_pool(); }
inline void h2d(void* dst, const void* src, size_t b) { wsCheck(ws_h2d(dst, src, b)); }
inline void d2h(void* dst, const void* src, size_t b) { wsCheck(ws_d2h(dst, src, b)); }
inline void d2d(void* dst, const void* src, size_t b) { wsCheck(ws_d2d(dst, src, b)); }
inline void gpuSync() { wsCheck(ws_gpu_sync()); }

// ---- tiered column storage (src/gpu.h:19-47)
inline void gpuSetVramLimit(int64_t bytes) { wsCheck(ws_set_vram_limit(bytes)); }
inline int64_t gpuVramUsed() { return ws_vram_used(); }
inline double gpuVramFill() { return ws_vram_fill(); }
inline int64_t gpuVramLimit() { return ws_vram_limit(); }
inline int64_t gpuVramFree() { return ws_vram_free(); }
inline void* placeColumn(void* host, size_t bytes, bool& mapped, bool hostOnly = false) {
  void* d = nullptr;
  int m = 0;
  wsCheck(ws_place_column(host, bytes, hostOnly ? 1 : 0, &d, &m));
  mapped = m != 0;
  return d;
}
inline void releaseColumn(void* dev, void* host, size_t bytes, bool mapped) {
  wsCheck(ws_release_column(dev, host, bytes, mapped ? 1 : 0));
}
inline void* vramAcquire(const void* host, size_t bytes) {
  void* d = nullptr;
  wsCheck(ws_vram_acquire(host, bytes, &d));
  return d;
}
inline void vramRelease(void* dev, size_t bytes) { wsCheck(ws_vram_release(dev, bytes)); }
inline void* hostMap(void* host, size_t bytes) {
  void* d = nullptr;
  wsCheck(ws_host_map(host, bytes, &d));
  return d;
}
inline void hostUnmap(void* host) { ws_host_unmap(host); }
// column-level UPDATE (src/gpu.h:24-41)
inline void* gpuPatchColumn(const void* oldDev, size_t bytes, int width, const int32_t* rows, const void* vals, int64_t m) {
  void* d = nullptr;
  wsCheck(ws_patch_column(oldDev, bytes, width, rows, vals, m, &d));
  return d;
}
struct GpuUpdate {  // the engine's, field for field (ws_update)
  int kind = 0;
  int64_t i0 = 0, add = 0, nul = 0, lo = 0, hi = 0;
  double d0 = 0, addD = 0;
  bool notNull = false;
  bool bad = false, sawNull = false;
  double mn = 0, mx = 0;
};
static_assert(sizeof(GpuUpdate) == sizeof(ws_update) && offsetof(GpuUpdate, i0) == offsetof(ws_update, i0) &&
                  offsetof(GpuUpdate, hi) == offsetof(ws_update, hi) && offsetof(GpuUpdate, addD) == offsetof(ws_update, add_d) &&
                  offsetof(GpuUpdate, notNull) == offsetof(ws_update, not_null) &&
                  offsetof(GpuUpdate, sawNull) == offsetof(ws_update, saw_null) && offsetof(GpuUpdate, mn) == offsetof(ws_update, mn) &&
                  offsetof(GpuUpdate, mx) == offsetof(ws_update, mx),
              "GpuUpdate and ws_update differ");
inline void* gpuUpdateColumn(const void* old, const void* src, int64_t n, int w, bool f64, const int32_t* rows, int64_t m,
                             GpuUpdate& u) {
  ws_update c{};
  c.kind = u.kind, c.i0 = u.i0, c.add = u.add, c.nul = u.nul, c.lo = u.lo, c.hi = u.hi, c.d0 = u.d0, c.add_d = u.addD;
  c.not_null = u.notNull ? 1 : 0;
  void* d = nullptr;
  wsCheck(ws_update_column(old, src, n, w, f64 ? 1 : 0, rows, m, &c, &d));
  u.bad = c.bad != 0, u.sawNull = c.saw_null != 0, u.mn = c.mn, u.mx = c.mx;
  return d;
}

// RAII temp device array (src/gpu.h:59-79)
template <class T>
struct DevVec {
  T* p = nullptr;
  int64_t n = 0;
  DevVec() = default;
  explicit DevVec(int64_t count) : n(count) { p = count ? (T*)tmpAlloc(sizeof(T) * count) : nullptr; }
  DevVec(T* q, int64_t count) : p(q), n(count) {}  // takes over a buffer returned by the C ABI
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
  DevVec(DevVec&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr, o.n = 0; }
  DevVec& operator=(DevVec&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p, n = o.n;
      o.p = nullptr, o.n = 0;
    }
    return *this;
  }
  ~DevVec() { reset(); }
  void reset() {
    if (p) tmpFree(p);
    p = nullptr, n = 0;
  }
  std::vector<T> download(int64_t count = -1) const {
    std::vector<T> v(count < 0 ? n : count);
    if (!v.empty()) d2h(v.data(), p, sizeof(T) * v.size());
    return v;
  }
};

// ---- compiled plans (src/jit.h)
using JitProgram = ws_jit_program;
enum JitFn { JF_NOKEYS = WS_JF_NOKEYS, JF_GROUPED = WS_JF_GROUPED, JF_DENSE = WS_JF_DENSE, JF_FLAG = WS_JF_FLAG, JF_FLAGM = WS_JF_FLAGM };
enum JitMode { JIT_OFF = WS_JIT_OFF, JIT_ON = WS_JIT_ON, JIT_SYNC = WS_JIT_SYNC };
inline JitMode jitMode() { return (JitMode)ws_jit_mode(); }
inline bool jitEnabled() { return jitMode() != JIT_OFF; }
inline void jitSetMode(JitMode m) { ws_jit_set_mode(m); }
inline void jitSetDefaultMode(JitMode m) { ws_jit_set_default_mode(m); }
inline void jitSetCacheDir(const std::string& dir) { wsCheck(ws_jit_set_cache_dir(dir.c_str())); }
inline const JitProgram* jitGet(const ExprEnv& env, int ncols, const AggPlan& plan, JitFn fn, const std::string& kind) {
  const ws_jit_program* p = nullptr;
  wsCheck(ws_jit_get((const ws_expr_env*)&env, ncols, (const ws_agg_plan*)&plan, fn, kind.c_str(), &p));
  return p;
}
inline bool progIsInt(const ExprEnv& env, Prog p) { return ws_prog_is_int((const ws_expr_env*)&env, *(const ws_prog*)&p) != 0; }
inline void jitBeginQuery(const std::string& sql) { ws_jit_begin_query(sql.c_str()); }
// src/jit.h:51-56
struct JitQueryInfo {
  int compiled = 0, hits = 0, fromDisk = 0, background = 0;
  double compileMs = 0;
  std::vector<int> ids;
};
inline JitQueryInfo jitEndQuery(double queryMs) {
  ws_jit_query_info i{};
  ws_jit_end_query(queryMs, &i);
  JitQueryInfo r;
  r.compiled = i.compiled, r.hits = i.hits, r.fromDisk = i.from_disk, r.background = i.background;
  r.compileMs = i.compile_ms;
  int n = 0;
  if (ws_jit_last_query_plans(nullptr, 0, &n) == WS_ERR_SIZE) {
    r.ids.resize((size_t)n);
    ws_jit_last_query_plans(r.ids.data(), n, &n);
  }
  return r;
}
inline std::string wsJitPlanText(int id, int field) {
  size_t need = 0;
  if (ws_jit_plan_text(id, field, nullptr, 0, &need) != WS_OK || need == 0) return "";
  std::string t(need, '\0');
  ws_jit_plan_text(id, field, t.data(), need, &need);
  t.resize(need - 1);
  return t;
}
// src/jit.h:61-73
struct PlanCacheRow {
  int id;
  std::string kind;
  std::string origin;  // "compiled" or "disk"
  double compileMs;
  int64_t execs;
  double avgMs, lastMs;
  size_t sourceBytes;
  std::string sql;
};
inline std::vector<PlanCacheRow> jitPlanCache() {
  std::vector<PlanCacheRow> rows;
  const int n = ws_jit_plan_cache_count();
  for (int i = 0; i < n; ++i) {
    ws_jit_info j{};
    if (ws_jit_plan_cache_row(i, &j) != WS_OK) continue;
    rows.push_back({j.id, wsJitPlanText(j.id, 0), j.from_disk ? "disk" : "compiled", j.compile_ms, j.execs,
                    j.execs ? j.total_ms / (double)j.execs : 0.0, j.last_ms, (size_t)j.source_bytes,
                    wsJitPlanText(j.id, 1)});
  }
  return rows;
}
inline std::string jitSourceOf(int id) { return wsJitPlanText(id, 2); }
inline void jitClearCache() { ws_jit_clear_cache(); }

// ---- aggregation (src/gpu.h:84-130)
class GpuAggregator {
 public:
  GpuAggregator(const AggPlan& plan, int64_t capacity, const DenseSpec* dense = nullptr) : naggs_(plan.naggs), nkeys_(plan.nkeys) {
    wsCheck(ws_agg_create((const ws_agg_plan*)&plan, capacity, (const ws_dense_spec*)dense, &h_));
  }
  ~GpuAggregator() { ws_agg_destroy(h_); }
  GpuAggregator(const GpuAggregator&) = delete;
  GpuAggregator& operator=(const GpuAggregator&) = delete;
  void addBatch(const ExprEnv& env, int ncols, int64_t n, const uint32_t* del) {
    wsCheck(ws_agg_add_batch(h_, (const ws_expr_env*)&env, ncols, n, del));
  }
  void run(const ExprEnv& env, const JitProgram* jit) { wsCheck(ws_agg_run(h_, (const ws_expr_env*)&env, jit)); }
  void runWindow(const ExprEnv& env, const JitProgram* jit) { wsCheck(ws_agg_run_window(h_, (const ws_expr_env*)&env, jit)); }
  int batches() const { return ws_agg_batches(h_); }
  int windows() const { return ws_agg_windows(h_); }
  int64_t rowsIn() const { return ws_agg_rows_in(h_); }
  bool dense() const { return ws_agg_is_dense(h_) != 0; }
  bool overflowed() {
    int o = 0;
    wsCheck(ws_agg_overflowed(h_, &o));
    return o != 0;
  }
  int64_t fetch(std::vector<double>& keys, std::vector<double>& accs) {
    int64_t g = 0;
    int rc = ws_agg_fetch(h_, 0, nullptr, nullptr, nullptr, &g);
    if (rc != WS_OK && rc != WS_ERR_SIZE) wsCheck(rc);
    keys.resize((size_t)g * nkeys_);
    accs.resize((size_t)g * naggs_);
    wsCheck(ws_agg_fetch(h_, g, keys.data(), accs.data(), nullptr, &g));
    hi_.assign(naggs_, 0);
    ws_agg_sum_high(h_, hi_.data());
    return g;
  }
  // Addition (no counterpart in gpu.h): groups [first, first + max) straight into pinned host memory
  // (keys [.][nkeys], exact [.][naggs][2]); status valid after the stream is synchronised.
  void fetchAsync(int64_t first, int64_t max, double* keys, int64_t* exact, ws_fetch_status* status) {
    wsCheck(ws_agg_fetch_async(h_, first, max, keys, exact, status));
  }
  std::vector<uint8_t> sumBitsSlots() const {
    std::vector<uint8_t> f(naggs_);
    ws_agg_sum_bits_slots(h_, f.data());
    return f;
  }
  const std::vector<int64_t>& sumHigh() const { return hi_; }
  int64_t compact(DevVec<double>& keys, DevVec<double>& accs) {
    double *k = nullptr, *a = nullptr;
    int64_t g = 0;
    wsCheck(ws_agg_compact(h_, &k, &a, &g));
    keys = DevVec<double>(k, g * nkeys_);
    accs = DevVec<double>(a, g * naggs_);
    return g;
  }
  int64_t capacity() const { return ws_agg_capacity(h_); }
  int64_t groupCount() {
    int64_t g = 0;
    wsCheck(ws_agg_group_count(h_, &g));
    return g;
  }

 private:
  ws_aggregator* h_ = nullptr;
  int naggs_, nkeys_;
  std::vector<int64_t> hi_;
};

// Addition (no counterpart in gpu.h): a query prepared once as a CUDA graph and rerun with new
// constants (ws_exec_*).  Results live in the executor's pinned memory until the next run.
class PreparedQuery {
 public:
  PreparedQuery(const AggPlan& plan, int64_t capacity, const DenseSpec* dense, const ExprEnv& env, int ncols,
                const std::vector<int64_t>& bn, const std::vector<const uint32_t*>& bdel,
                const std::vector<ColView>& bcols, const JitProgram* jit, int64_t maxGroups) {
    wsCheck(ws_exec_create((const ws_agg_plan*)&plan, capacity, (const ws_dense_spec*)dense,
                           (const ws_expr_env*)&env, ncols, (int)bn.size(), bn.data(), bdel.data(),
                           (const ws_col_view*)bcols.data(), jit, maxGroups, &h_));
  }
  ~PreparedQuery() { ws_exec_destroy(h_); }
  PreparedQuery(const PreparedQuery&) = delete;
  PreparedQuery& operator=(const PreparedQuery&) = delete;
  void run(const ExprEnv& env) { wsCheck(ws_exec_run(h_, (const ws_expr_env*)&env)); }
  // after gpuSync(): keys [g][nkeys], exact [g][naggs][2], status (groups, overflow, error)
  void results(const double** keys, const int64_t** exact, const ws_fetch_status** status) {
    wsCheck(ws_exec_results(h_, keys, exact, status));
  }

 private:
  ws_executor* h_ = nullptr;
};

// ---- selection / gathers (src/gpu.h:132-143, :170-172)
inline int64_t gpuSelect(const ExprEnv& env, bool hasWhere, Prog where, int64_t n, const uint32_t* del, int32_t* outIdx,
                         const JitProgram* jit = nullptr) {
  int64_t c = 0;
  wsCheck(ws_select((const ws_expr_env*)&env, hasWhere, *(const ws_prog*)&where, n, del, outIdx, jit, &c));
  return c;
}
inline int64_t gpuSelectMulti(const ExprEnv& env, bool hasWhere, Prog where, const std::vector<int64_t>& bn,
                              const std::vector<const uint32_t*>& bdel, const std::vector<ColView>& bcols, int ncols,
                              DevVec<int32_t>& outIdx, std::vector<int64_t>& perBatch, const JitProgram* jit = nullptr) {
  perBatch.assign(bn.size(), 0);
  int32_t* idx = nullptr;
  int64_t c = 0;
  wsCheck(ws_select_multi((const ws_expr_env*)&env, hasWhere, *(const ws_prog*)&where, (int)bn.size(),
                          (const int64_t*)bn.data(), bdel.data(), (const ws_col_view*)bcols.data(), ncols, &idx,
                          (int64_t*)perBatch.data(), jit, &c));
  outIdx = DevVec<int32_t>(idx, c);
  return c;
}
template <class PType>
inline void gpuGatherMulti(const std::vector<ColView>& src, const std::vector<int64_t>& boff, PType t, int esize,
                           const int32_t* idx, int64_t m, void* dst) {
  wsCheck(ws_gather_multi((const ws_col_view*)src.data(), (const int64_t*)boff.data(), (int)src.size(), (int)t, esize, idx, m, dst));
}
template <class PType>
inline void gpuGather(const void* src, PType t, const int32_t* idx, int64_t m, void* dst) {
  wsCheck(ws_gather(src, (int)t, idx, m, dst));
}

// ---- joins (src/gpu.h:178-186)
inline int64_t gpuHashJoinParts(ColView buildKey, const std::vector<int64_t>& bOff, ColView probeKey,
                                const std::vector<int64_t>& pOff, DevVec<int32_t>& outBuild, DevVec<int32_t>& outProbe,
                                std::vector<int64_t>* outOff) {
  int32_t *ob = nullptr, *op = nullptr;
  int64_t m = 0;
  std::vector<int64_t> off(pOff.size(), 0);
  wsCheck(ws_hash_join_parts(*(const ws_col_view*)&buildKey, (const int64_t*)bOff.data(), (int)bOff.size() - 1,
                             *(const ws_col_view*)&probeKey, (const int64_t*)pOff.data(), (int)pOff.size() - 1, &ob, &op,
                             (int64_t*)off.data(), &m));
  outBuild = DevVec<int32_t>(ob, m);
  outProbe = DevVec<int32_t>(op, m);
  if (outOff) *outOff = off;
  return m;
}
inline int64_t gpuHashJoin(ColView buildKey, int64_t nb, ColView probeKey, int64_t np, DevVec<int32_t>& outBuild,
                           DevVec<int32_t>& outProbe) {
  return gpuHashJoinParts(buildKey, {0, nb}, probeKey, {0, np}, outBuild, outProbe, nullptr);
}
inline int64_t gpuHashJoinOuter(ColView buildKey, int64_t nb, ColView probeKey, int64_t np, DevVec<int32_t>& outBuild,
                                DevVec<int32_t>& outProbe, bool full) {
  int32_t *ob = nullptr, *op = nullptr;
  int64_t m = 0;
  wsCheck(ws_hash_join_outer(*(const ws_col_view*)&buildKey, nb, *(const ws_col_view*)&probeKey, np, full ? 1 : 0, &ob,
                             &op, &m));
  outBuild = DevVec<int32_t>(ob, m);
  outProbe = DevVec<int32_t>(op, m);
  return m;
}
inline int64_t gpuCrossJoin(int64_t na, int64_t nb, DevVec<int32_t>& outA, DevVec<int32_t>& outB) {
  int32_t *a = nullptr, *b = nullptr;
  int64_t m = 0;
  wsCheck(ws_cross_join(na, nb, &a, &b, &m));
  outA = DevVec<int32_t>(a, m);
  outB = DevVec<int32_t>(b, m);
  return m;
}
inline void gpuKeyBitmap(ColView key, int64_t n, int64_t lo, int64_t nbits, uint32_t* bits) {
  wsCheck(ws_key_bitmap(*(const ws_col_view*)&key, n, lo, nbits, bits));
}
inline void gpuSetBits(uint32_t* bits, const int32_t* idx, int64_t m) { wsCheck(ws_set_bits(bits, idx, m)); }

// ---- codes, NULL-aware gathers, evaluation at rows (src/gpu.h:145-172, :190-195)
inline void gpuRemapCodes(const int32_t* in, int64_t n, const int32_t* map, int64_t mapN, int32_t* out) {
  wsCheck(ws_remap_codes(in, n, map, mapN, out));
}
inline void gpuBitsToDouble(const double* src, int64_t n, double* dst) { wsCheck(ws_bits_to_double(src, n, dst)); }
template <class PType>
inline void gpuGatherNull(const void* src, PType t, const int32_t* idx, int64_t m, void* dst) {
  wsCheck(ws_gather_null(src, (int)t, idx, m, dst));
}
inline void gpuGatherBytes(const void* src, int esize, const int32_t* idx, int64_t m, void* dst, bool nulls) {
  wsCheck(ws_gather_bytes(src, esize, idx, m, dst, nulls ? 1 : 0));
}
template <class PType>
inline void gpuGatherEnc(const ColView& v, PType t, const int32_t* idx, int64_t m, void* dst) {
  wsCheck(ws_gather_enc(*(const ws_col_view*)&v, (int)t, idx, m, dst));
}
inline void gpuEvalAt(const ExprEnv& env, Prog prog, const int32_t* idx, int64_t m, double* out) {
  wsCheck(ws_eval_at((const ws_expr_env*)&env, WS_MAX_COLS, *(const ws_prog*)&prog, idx, m, out));
}
inline void gpuEvalAtInt(const ExprEnv& env, Prog prog, const int32_t* idx, int64_t m, int64_t* out) {
  wsCheck(ws_eval_at_int((const ws_expr_env*)&env, WS_MAX_COLS, *(const ws_prog*)&prog, idx, m, out));
}

// ---- distinct values, bitmaps, temp-table columns (src/gpu.h:150-167)
inline std::vector<int64_t> gpuDistinctInts(const ExprEnv& env, Prog prog, const int32_t* idx, int64_t m, int64_t base,
                                            int64_t span) {
  std::vector<int64_t> out((size_t)std::min<int64_t>(std::max<int64_t>(std::min(span, m), 0), 1 << 16));
  int64_t n = 0;
  int rc = ws_distinct_ints((const ws_expr_env*)&env, WS_MAX_COLS, *(const ws_prog*)&prog, idx, m, base, span, out.data(),
                            (int64_t)out.size(), &n);
  if (rc == WS_ERR_SIZE) {
    out.resize((size_t)n);
    rc = ws_distinct_ints((const ws_expr_env*)&env, WS_MAX_COLS, *(const ws_prog*)&prog, idx, m, base, span, out.data(),
                          (int64_t)out.size(), &n);
  }
  wsCheck(rc);
  out.resize((size_t)n);
  return out;
}
inline uint32_t* gpuBitsFromColumn(const void* col, int out, int64_t n, int64_t base, int64_t nbits, bool* sawNull) {
  uint32_t* bits = nullptr;
  int nul = 0;
  wsCheck(ws_bits_from_column(col, out, n, base, nbits, &bits, &nul));
  if (sawNull) *sawNull = nul != 0;
  return bits;
}
struct TempColSpec {  // the engine's, field for field (ws_temp_col_spec)
  int8_t src = 0;
  int idx = 0, hi = -1, cnt = -1;
  uint8_t kind = 0;
  uint8_t keyInt = 0, sumBits = 0;
  uint8_t out = 2;
  double div = 1;
  double mul = 1;
};
static_assert(sizeof(TempColSpec) == sizeof(ws_temp_col_spec) && offsetof(TempColSpec, idx) == offsetof(ws_temp_col_spec, idx) &&
                  offsetof(TempColSpec, cnt) == offsetof(ws_temp_col_spec, cnt) &&
                  offsetof(TempColSpec, kind) == offsetof(ws_temp_col_spec, kind) &&
                  offsetof(TempColSpec, out) == offsetof(ws_temp_col_spec, out) &&
                  offsetof(TempColSpec, div) == offsetof(ws_temp_col_spec, div) &&
                  offsetof(TempColSpec, mul) == offsetof(ws_temp_col_spec, mul),
              "TempColSpec and ws_temp_col_spec differ");
inline void* gpuTempColumn(const double* keys, int nk, const double* accs, int na, int64_t g, const TempColSpec& s, double& mn,
                           double& mx) {
  void* col = nullptr;
  wsCheck(ws_temp_column(keys, nk, accs, na, g, (const ws_temp_col_spec*)&s, &col, &mn, &mx));
  return col;
}

// ---- ORDER BY (src/gpu.h:197-199)
inline DevVec<int32_t> gpuSortPerm(const std::vector<std::pair<const double*, bool>>& keys, int64_t m) {
  std::vector<const double*> k;
  std::vector<int> d;
  for (auto& [p, desc] : keys) k.push_back(p), d.push_back(desc ? 1 : 0);
  int32_t* perm = nullptr;
  wsCheck(ws_sort_perm(k.data(), d.data(), (int)k.size(), m, &perm));
  return DevVec<int32_t>(perm, m);
}
inline void gpuMapRank(double* keys, const int32_t* rank, int64_t m) { wsCheck(ws_map_rank(keys, rank, m)); }
template <class PType>
inline std::vector<int32_t> gpuSortPermHost(const void* hostCol, PType t, int64_t n) {
  std::vector<int32_t> perm((size_t)std::max<int64_t>(n, 0));
  if (n > 0) wsCheck(ws_sort_perm_host(hostCol, (int)t, n, perm.data()));
  return perm;
}

}  // namespace gdb
