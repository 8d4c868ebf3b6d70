// Native request loop: prepared GROUP BY queries served by a pool of host threads, each with its own
// CUDA stream (the admitted queries' kernels overlap on the device), admitted in arrival order as a
// slot frees and while the HBM footprint of the queries in flight stays within the budget.  With
// estimator weights, a query whose plain-rule table is large is sized from the learned estimate (GPU
// sketch + GPU MLP); the plain rule's overflow retry stays the fallback.  No counterpart in the
// reference, whose connections each run their query synchronously (src/server.cpp).
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <thread>

#include "ws_b200.h"
#include "ws_internal.h"

namespace {

double nowS() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// HyperLogLog estimate of a sketch (Flajolet et al. 2007; linear counting for small cardinalities)
double hllEstimate(const std::vector<uint32_t>& regs) {
  const double m = (double)regs.size();
  const double alpha = 0.7213 / (1 + 1.079 / m);
  double sum = 0;
  int zeros = 0;
  for (uint32_t r : regs) {
    sum += std::ldexp(1.0, -(int)r);
    zeros += r == 0;
  }
  double e = alpha * m * m / sum;
  if (e <= 2.5 * m && zeros) e = m * std::log(m / zeros);
  return e;
}

// The estimator's nine inputs (the same definition as the Python package's features())
void features(const std::vector<uint32_t>& regs, int64_t sampled, int64_t passing, int64_t total, double keyRange,
              float* x) {
  const double est = hllEstimate(regs);
  const double scale = (double)total / (double)std::max<int64_t>(sampled, 1);
  const double kr = keyRange > 0 ? keyRange : std::ldexp(1.0, 63);
  const double naive = std::min({est * scale, (double)passing * scale, kr});
  int zeros = 0;
  for (uint32_t r : regs) zeros += r == 0;
  x[0] = (float)std::log2(1 + est);
  x[1] = (float)std::log2(1 + (double)passing);
  x[2] = (float)std::log2(1 + (double)sampled);
  x[3] = (float)std::log2(1 + (double)total);
  x[4] = (float)std::min(std::log2(1 + kr), 64.0);
  x[5] = (float)(est / (double)std::max<int64_t>(passing, 1));
  x[6] = (float)((double)passing / (double)std::max<int64_t>(sampled, 1));
  x[7] = (float)((double)zeros / (double)regs.size());
  x[8] = (float)std::log2(1 + naive);
}

int64_t pow2AtLeast(double x, int64_t lo) {
  int64_t c = lo;
  while ((double)c < x) c <<= 1;
  return c;
}

int64_t grow(int64_t cap, int64_t groups) {  // after an overflow: pow2 >= max(4 cap, 4 groups)
  const int64_t want = std::max(cap * 4, groups * 4);
  int64_t c = 1;
  while (c < want) c <<= 1;
  return c;
}

void checkRc(int rc) {
  if (rc) throw ws::Error(ws_last_error(), rc);
}

bool pinnedHost(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost && at.devicePointer;
}

// One query on the calling thread's stream.  Results into pinned host arrays (keys / exact, no accs)
// take the one-sync form: run, compaction and the kernel that writes the groups into host memory are
// queued back to back, and the thread waits once; otherwise the engine's sequence (overflow check,
// group count, compaction, copies), which waits at each step.
void serveOne(ws_serve_query& q, const ws_estimator_weights* w, ws_fetch_status* st) {
  int64_t cap = q.cap_plain;
  if (w && cap > (1 << 16)) {
    std::vector<uint32_t> regs(1u << 12);
    int64_t sampled = 0, passing = 0, total = 0;
    for (int b = 0; b < q.nb; ++b) total += q.bn[b];
    checkRc(ws_hll_sketch(q.env, q.ncols, q.plan, q.nb, q.bn, q.bdel, q.bcols, 12, 1 << 18, regs.data(), &sampled,
                          &passing));
    float x[9], xn[9], y = 0;
    features(regs, sampled, passing, total, q.key_range, x);
    for (int i = 0; i < 9; ++i) xn[i] = (x[i] - w->mean[i]) / w->std[i];
    checkRc(ws_mlp_infer(xn, 1, 9, w->hidden, w->w1, w->b1, w->w2, w->b2, w->w3, w->b3, &y));
    const double pred = std::exp2((double)x[8] + (double)y) - 1;
    cap = std::min(cap, pow2AtLeast(2 * pred * w->margin, 1024));
  }
  q.runs = 0;
  for (;;) {
    ++q.runs;
    ws_aggregator* a = nullptr;
    checkRc(ws_agg_create(q.plan, cap, nullptr, &a));
    int rc = ws_agg_add_batches(a, q.ncols, q.nb, q.bn, q.bdel, q.bcols);
    if (!rc) rc = ws_agg_run(a, q.env, q.jit);
    if (st) {
      if (!rc) rc = ws_agg_fetch_async(a, q.max_groups, q.keys, q.exact, st);
      if (!rc) rc = ws_gpu_sync();
      ws_agg_destroy(a);
      checkRc(rc);
      if (st->error) throw ws::Error("serve: the aggregation raised an error flag", st->error);
      if (st->overflow) {
        cap = grow(cap, st->groups);
        continue;
      }
      if (st->groups > q.max_groups)
        throw ws::Error("output buffer too small for " + std::to_string(st->groups) + " groups", WS_ERR_SIZE);
      q.groups = st->groups;
      q.cap_used = cap;
      return;
    }
    int ovf = 0;
    if (!rc) rc = ws_agg_overflowed(a, &ovf);
    if (!rc && ovf) {
      int64_t g = 0;
      rc = ws_agg_group_count(a, &g);
      ws_agg_destroy(a);
      checkRc(rc);
      cap = grow(cap, g);
      continue;
    }
    int64_t g = 0;  // without result arrays the groups stay on the device (compacted, not downloaded)
    const bool keep = q.keys || q.accs || q.exact;
    if (!rc) rc = ws_agg_fetch(a, keep ? q.max_groups : INT64_MAX, q.keys, q.accs, q.exact, &g);
    ws_agg_destroy(a);
    checkRc(rc);
    q.groups = g;
    q.cap_used = cap;
    return;
  }
}

}  // namespace

extern "C" {

int ws_serve(ws_serve_query* queries, int n, int slots, int64_t hbm_budget, const ws_estimator_weights* est,
             double* wall_s) {
  return ws::guardedCall([&] {
    if (slots < 1 || slots > 256) throw ws::Error("serve: 1 to 256 slots", WS_ERR_ARG);
    ws_gpu_init();
    std::mutex mu;
    std::condition_variable cv;
    int64_t inFlight = 0;
    std::atomic<int> next{0}, failed{0};
    std::string firstError;
    int firstCode = 0;
    const double t0 = nowS();
    auto worker = [&] {
      cudaStream_t s = nullptr;
      if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        failed = 1;
        return;
      }
      ws_set_stream(s);
      ws_fetch_status* st = nullptr;  // this worker's fetch status (pinned, for the one-sync form)
      if (cudaHostAlloc((void**)&st, sizeof(ws_fetch_status), cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        st = nullptr;
        failed = 1;
      }
      for (;;) {
        const int i = next++;
        if (i >= n || failed) break;
        ws_serve_query& q = queries[i];
        const double wait = q.arrival_s - (nowS() - t0);  // the query has not arrived yet
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        {
          std::unique_lock<std::mutex> l(mu);  // admission by HBM footprint
          cv.wait(l, [&] { return inFlight == 0 || inFlight + q.footprint <= hbm_budget; });
          inFlight += q.footprint;
        }
        q.start_s = nowS() - t0;
        try {
          const bool oneSync = (q.keys || !q.plan->nkeys) && q.exact && !q.accs && pinnedHost(q.exact) &&
                               (!q.keys || pinnedHost(q.keys));
          serveOne(q, est, oneSync ? st : nullptr);
        } catch (const ws::Error& e) {
          std::lock_guard<std::mutex> l(mu);
          if (!failed++) firstError = e.what(), firstCode = e.code;
        }
        q.finish_s = nowS() - t0;
        {
          std::lock_guard<std::mutex> l(mu);
          inFlight -= q.footprint;
        }
        cv.notify_all();
      }
      ws_set_stream(nullptr);
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
      if (st) cudaFreeHost(st);
    };
    std::vector<std::thread> th;
    for (int k = 0; k < slots; ++k) th.emplace_back(worker);
    for (auto& t : th) t.join();
    if (wall_s) *wall_s = nowS() - t0;
    if (failed) throw ws::Error(firstError.empty() ? "serve: a worker could not start" : firstError,
                                firstCode ? firstCode : WS_ERR_INTERNAL);
  });
}

}  // extern "C"
