// Harness around the reference's own GPU operators (Warpstore src/gpu.cu and src/jit.cu, built for
// sm_100a from their sources by oracle/build_ref.py) — TEST INFRASTRUCTURE ONLY: a second parity
// checker that runs the reference on the same inputs, and its timing for comparison.  Only tests/
// call it.
//
// By default the operators run the engine's production path: each aggregation and selection first
// gets its compiled plan (jitGet in JIT_SYNC mode: NVRTC compiles before the first run, outside the
// timed region) and hands it to the operator, as src/engine_select.cpp:1379-1392 and
// src/engine_core.h:4372-4378 do.  wsref_set_compiled(0) selects the interpreted kernels instead (the
// engine with codegen OFF).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "gpu.h"
#include "jit.h"

using namespace gdb;

static thread_local char gErr[512];
static bool gCompiled = true;                // run compiled plans (the engine's production path)
static thread_local int gLastCompiled = 0;  // the last aggregation / selection ran a compiled plan

template <class F>
static int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    strncpy(gErr, e.what(), sizeof gErr - 1);
    return 1;
  }
}

// The compiled plan the engine would run for an aggregation or a filter (nullptr: interpreted).
static const JitProgram* aggPlanFor(const ExprEnv& env, int ncols, const AggPlan& plan, const DenseSpec* dense) {
  if (!gCompiled) return nullptr;
  jitSetMode(JIT_SYNC);
  const JitFn fn = !plan.nkeys ? JF_NOKEYS : (dense && dense->G) ? JF_DENSE : JF_GROUPED;
  return jitGet(env, ncols, plan, fn, "harness aggregate");
}
static const JitProgram* filterPlanFor(const ExprEnv& env, int ncols, bool hasWhere, Prog where) {
  if (!gCompiled || !hasWhere) return nullptr;
  jitSetMode(JIT_SYNC);
  AggPlan fp;
  fp.hasWhere = true;
  fp.where = where;
  return jitGet(env, ncols, fp, JF_FLAGM, "harness filter");
}

extern "C" {

const char* wsref_error() { return gErr; }

int wsref_init() {
  return guard([] {
    gpuInit();
    jitSetDefaultMode(JIT_SYNC);
  });
}
int wsref_set_compiled(int on) {
  gCompiled = on != 0;
  return 0;
}
int wsref_last_compiled() { return gLastCompiled; }

// Result of the last wsref_aggregate on this thread, copied out by wsref_take.
static thread_local std::vector<double> gKeys, gAccs;
static thread_local std::vector<int64_t> gHi;

// GpuAggregator over batches (views bcols[b * ncols + c]): one aggregation, groups kept in the engine
// format for wsref_take; *ngroups = their number.  *ms: CUDA-event time of run() + overflowed() on the
// default per-thread stream.
int wsref_aggregate(const ExprEnv* envIn, int ncols, const AggPlan* plan, const DenseSpec* dense, int64_t cap, int nb,
                    const int64_t* bn, const uint32_t* const* bdel, const ColView* bcols, int64_t* ngroups,
                    int* overflow, float* ms) {
  return guard([&] {
    std::vector<uint8_t> envBuf(sizeof(ExprEnv));
    ExprEnv* env = (ExprEnv*)envBuf.data();
    memcpy(env, envIn, sizeof(ExprEnv));
    if (nb > 0)
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[c];
    const JitProgram* jit = aggPlanFor(*env, ncols, *plan, dense);
    gLastCompiled = jit != nullptr;
    GpuAggregator agg(*plan, cap, dense);
    for (int b = 0; b < nb; ++b) {
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[(int64_t)b * ncols + c];
      agg.addBatch(*env, ncols, bn[b], bdel ? bdel[b] : nullptr);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    agg.run(*env, jit);
    cudaEventRecord(e1, cudaStreamPerThread);
    *overflow = agg.overflowed() ? 1 : 0;
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    gKeys.clear();
    gAccs.clear();
    gHi.assign(plan->naggs, 0);
    if (*overflow) {
      *ngroups = agg.groupCount();
      return;
    }
    *ngroups = agg.fetch(gKeys, gAccs);
    const auto& hi = agg.sumHigh();
    for (int i = 0; i < plan->naggs && i < (int)hi.size(); ++i) gHi[i] = hi[i];
  });
}

// GpuAggregator over batches leaving the groups on the device, column-major (GpuAggregator::compact);
// *keys / *accs are freed with wsref_free.  With *overflow set nothing is compacted.
int wsref_aggregate_compact(const ExprEnv* envIn, int ncols, const AggPlan* plan, const DenseSpec* dense, int64_t cap,
                            int nb, const int64_t* bn, const uint32_t* const* bdel, const ColView* bcols,
                            int64_t* ngroups, int* overflow, double** keys, double** accs, float* ms) {
  return guard([&] {
    std::vector<uint8_t> envBuf(sizeof(ExprEnv));
    ExprEnv* env = (ExprEnv*)envBuf.data();
    memcpy(env, envIn, sizeof(ExprEnv));
    if (nb > 0)
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[c];
    const JitProgram* jit = aggPlanFor(*env, ncols, *plan, dense);
    gLastCompiled = jit != nullptr;
    GpuAggregator agg(*plan, cap, dense);
    for (int b = 0; b < nb; ++b) {
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[(int64_t)b * ncols + c];
      agg.addBatch(*env, ncols, bn[b], bdel ? bdel[b] : nullptr);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    agg.run(*env, jit);
    cudaEventRecord(e1, cudaStreamPerThread);
    *overflow = agg.overflowed() ? 1 : 0;
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *keys = *accs = nullptr;
    if (*overflow) {
      *ngroups = agg.groupCount();
      return;
    }
    DevVec<double> k, a;
    *ngroups = agg.compact(k, a);
    *keys = k.p;
    *accs = a.p;
    k.p = nullptr;
    a.p = nullptr;
  });
}

// Copies the kept groups (keys [g][nkeys], accs [g][naggs], sum high words [naggs]).
int wsref_take(double* keys, double* accs, int64_t* sumHigh) {
  return guard([&] {
    if (keys && !gKeys.empty()) memcpy(keys, gKeys.data(), gKeys.size() * 8);
    if (accs && !gAccs.empty()) memcpy(accs, gAccs.data(), gAccs.size() * 8);
    if (sumHigh && !gHi.empty()) memcpy(sumHigh, gHi.data(), gHi.size() * 8);
  });
}

// Inner hash join (gpuHashJoin); pairs copied to the host arrays when m <= maxm.
int wsref_hash_join(ColView bk, int64_t nb, ColView pk, int64_t np, int64_t maxm, int64_t* m, int32_t* ob, int32_t* op,
                    float* ms) {
  return guard([&] {
    DevVec<int32_t> b, p;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    *m = gpuHashJoin(bk, nb, pk, np, b, p);
    cudaEventRecord(e1, cudaStreamPerThread);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (*m <= maxm && *m > 0) {
      d2h(ob, b.p, 4 * *m);
      d2h(op, p.p, 4 * *m);
    }
  });
}

// Row selection over batches (gpuSelectMulti); indices copied to idx when m <= maxm.
int wsref_select_multi(const ExprEnv* envIn, int hasWhere, Prog where, int nb, const int64_t* bn,
                       const uint32_t* const* bdel, const ColView* bcols, int ncols, int64_t maxm, int64_t* m, int32_t* idx,
                       int64_t* perBatch) {
  return guard([&] {
    std::vector<int64_t> n(bn, bn + nb);
    std::vector<const uint32_t*> d(nb, nullptr);
    if (bdel)
      for (int b = 0; b < nb; ++b) d[b] = bdel[b];
    std::vector<ColView> cols(bcols, bcols + (size_t)nb * ncols);
    DevVec<int32_t> out;
    std::vector<int64_t> per;
    const JitProgram* jit = filterPlanFor(*envIn, ncols, hasWhere != 0, where);
    gLastCompiled = jit != nullptr;
    *m = gpuSelectMulti(*envIn, hasWhere != 0, where, n, d, cols, ncols, out, per, jit);
    for (int b = 0; b < nb; ++b) perBatch[b] = per[b];
    if (*m <= maxm && *m > 0) d2h(idx, out.p, 4 * *m);
  });
}

// dst[j] = src[idx[j]] (gpuGather), all device pointers; *ms: CUDA-event time.
int wsref_gather(const void* src, int ptype, const int32_t* idx, int64_t m, void* dst, float* ms) {
  return guard([&] {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    gpuGather(src, (PType)ptype, idx, m, dst);
    cudaEventRecord(e1, cudaStreamPerThread);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

// Inner hash join leaving the pairs on the device (the engine's use): *ob / *op are cudaMallocAsync'd
// on the per-thread stream (free with wsref_free).
int wsref_hash_join_dev(ColView bk, int64_t nb, ColView pk, int64_t np, int64_t* m, int32_t** ob, int32_t** op, float* ms) {
  return guard([&] {
    DevVec<int32_t> b, p;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    *m = gpuHashJoin(bk, nb, pk, np, b, p);
    cudaEventRecord(e1, cudaStreamPerThread);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ob = b.p;
    *op = p.p;
    b.p = nullptr;
    p.p = nullptr;
  });
}

int wsref_free(void* p) {
  return guard([&] { tmpFree(p); });
}

// Row selection leaving the indices on the device.
int wsref_select_multi_dev(const ExprEnv* envIn, int hasWhere, Prog where, int nb, const int64_t* bn,
                           const uint32_t* const* bdel, const ColView* bcols, int ncols, int64_t* m, int32_t** idx,
                           float* ms) {
  return guard([&] {
    std::vector<int64_t> n(bn, bn + nb);
    std::vector<const uint32_t*> d(nb, nullptr);
    if (bdel)
      for (int b = 0; b < nb; ++b) d[b] = bdel[b];
    std::vector<ColView> cols(bcols, bcols + (size_t)nb * ncols);
    DevVec<int32_t> out;
    std::vector<int64_t> per;
    const JitProgram* jit = filterPlanFor(*envIn, ncols, hasWhere != 0, where);
    gLastCompiled = jit != nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    *m = gpuSelectMulti(*envIn, hasWhere != 0, where, n, d, cols, ncols, out, per, jit);
    cudaEventRecord(e1, cudaStreamPerThread);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *idx = out.p;
    out.p = nullptr;
  });
}

}  // extern "C"
