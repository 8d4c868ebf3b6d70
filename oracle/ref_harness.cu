// Harness around the reference's own GPU operators (Warpstore src/gpu.cu, built for sm_100a from its
// sources by oracle/build_ref.py) — TEST INFRASTRUCTURE ONLY: a second parity checker that runs the
// reference on the same inputs, and its timing for comparison.  Only tests/ call it.
//
// The reference's runtime-compiled plans (src/jit.cu) need a build-generated header and are not built;
// its operators run their ahead-of-time kernels with the bytecode interpreter (jit = nullptr), the
// engine's path with codegen OFF.  jitLaunch is therefore never reached (stub below).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "gpu.h"
#include "jit.h"

namespace gdb {
void jitLaunch(const JitProgram*, JitFn, unsigned, unsigned, size_t, void**) {
  throw SqlError("reference harness: compiled plans are not built", 1105);
}
}  // namespace gdb

using namespace gdb;

static thread_local char gErr[512];

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

extern "C" {

const char* wsref_error() { return gErr; }

int wsref_init() { return guard([] { gpuInit(); }); }

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
    GpuAggregator agg(*plan, cap, dense);
    for (int b = 0; b < nb; ++b) {
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[(int64_t)b * ncols + c];
      agg.addBatch(*env, ncols, bn[b], bdel ? bdel[b] : nullptr);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    agg.run(*env, nullptr);
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
    GpuAggregator agg(*plan, cap, dense);
    for (int b = 0; b < nb; ++b) {
      for (int c = 0; c < ncols; ++c) env->cols[c] = bcols[(int64_t)b * ncols + c];
      agg.addBatch(*env, ncols, bn[b], bdel ? bdel[b] : nullptr);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    agg.run(*env, nullptr);
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
    *m = gpuSelectMulti(*envIn, hasWhere != 0, where, n, d, cols, ncols, out, per, nullptr);
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
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, cudaStreamPerThread);
    *m = gpuSelectMulti(*envIn, hasWhere != 0, where, n, d, cols, ncols, out, per, nullptr);
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
