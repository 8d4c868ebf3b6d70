// Native request loop: prepared GROUP BY queries served by a pool of host threads, each with its own
// CUDA stream (the admitted queries' kernels overlap on the device), admitted in arrival order as a
// slot frees and while the HBM footprint of the queries in flight stays within the budget.  With
// estimator weights, a query whose plain-rule table is large is sized from the learned estimate (GPU
// sketch + GPU MLP); the plain rule's overflow retry stays the fallback.  No counterpart in the
// reference, whose connections each run their query synchronously (src/server.cpp).
#include <algorithm>
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

// The distinct values D of a population of equally frequent values whose sample of s rows shows d:
// the root of D (1 - exp(-s / D)) = d by bisection on log D; infinite when d is within 5 % of s (the
// sketch's error cannot tell such a sample from one of distinct rows).
double uniformDistinct(double d, double s) {
  if (d <= 0) return 0;
  if (d >= 0.95 * s) return HUGE_VAL;
  double lo = d, hi = d * std::ldexp(1.0, 60);
  for (int i = 0; i < 100; ++i) {
    const double mid = std::sqrt(lo * hi);
    if (mid * -std::expm1(-s / mid) < d) lo = mid;
    else hi = mid;
  }
  return hi;
}

// The estimator's ten inputs (the same definition as the Python package's features())
constexpr int kGroupFeatures = 10;
void features(const std::vector<uint32_t>& regs, int64_t sampled, int64_t passing, int64_t total, double keyRange,
              float* x) {
  const double est = hllEstimate(regs);
  const double scale = (double)total / (double)std::max<int64_t>(sampled, 1);
  const double kr = keyRange > 0 ? keyRange : std::ldexp(1.0, 63);
  const double scaled = std::min({est * scale, (double)passing * scale, kr});
  const double naive = std::min(uniformDistinct(est, (double)passing), scaled);
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
  x[8] = (float)std::log2(1 + scaled);
  x[9] = (float)std::log2(1 + naive);
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

uint64_t mix64h(uint64_t z) {  // splitmix64 finalizer
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Order-independent digest of delivered groups: the sum over groups of a hash of the group's key bits
// and exact words, DOUBLE SUM slots left out (their last bits depend on the order of the additions);
// those are added up separately.
void digest(const ws_agg_plan& plan, const double* keys, const int64_t* exact, int64_t rows, ws_serve_query& q) {
  const int nk = plan.nkeys, na = plan.naggs;
  for (int64_t r = 0; r < rows; ++r) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int k = 0; k < nk; ++k) {
      uint64_t b;
      std::memcpy(&b, keys + r * nk + k, 8);
      h = mix64h(h ^ b);
    }
    const int64_t* x = exact + r * na * 2;
    for (int a = 0; a < na; ++a) {
      if (plan.ops[a] == WS_AGG_SUM && !plan.aggInt[a]) {
        double d;
        std::memcpy(&d, x + 2 * a, 8);
        q.fsum += d;
        continue;
      }
      h = mix64h(h ^ (uint64_t)x[2 * a]);
      h = mix64h(h ^ (uint64_t)x[2 * a + 1]);
    }
    q.checksum += h;
  }
}

// A worker thread's result buffers for queries without result arrays (arena mode): pinned, delivered
// range by range, in the one-sync form; pageable, grown to the largest result, otherwise.
struct Arena {
  uint8_t* pinned = nullptr;
  int64_t bytes = 0;
  std::vector<uint8_t> host;
};

void growTo(std::vector<uint8_t>& v, size_t bytes) {
  if (v.size() < bytes) v.resize(bytes);
}

// One query on the calling thread's stream.
//  one-sync form (st != null): run, compaction and the kernel that writes the groups into pinned host
//    memory are queued back to back and the thread waits once per run (per range for results larger
//    than the arena);
//  otherwise the engine's sequence: overflow check, group count, compaction, copies, each a wait.
// The query's first hash table capacity: the plain rule's, or for a large table the learned estimate.
int64_t initialCap(const ws_serve_query& q, const ws_serve_options& o) {
  const ws_estimator_weights* w = o.est;
  int64_t cap = q.cap_plain;
  if (w && cap > (1 << 16)) {
    std::vector<uint32_t> regs(1u << 12);
    int64_t sampled = 0, passing = 0, total = 0;
    for (int b = 0; b < q.nb; ++b) total += q.bn[b];
    checkRc(ws_hll_sketch(q.env, q.ncols, q.plan, q.nb, q.bn, q.bdel, q.bcols, 12, 1 << 18, regs.data(), &sampled,
                          &passing));
    float x[kGroupFeatures], xn[kGroupFeatures], y = 0;
    features(regs, sampled, passing, total, q.key_range, x);
    for (int i = 0; i < kGroupFeatures; ++i) xn[i] = (x[i] - w->mean[i]) / w->std[i];
    checkRc(ws_mlp_infer(xn, 1, kGroupFeatures, w->hidden, w->w1, w->b1, w->w2, w->b2, w->w3, w->b3, &y));
    // log2(1 + groups) floored at log2(1 + 1024), the smallest capacity (as estimator.Model.gated)
    const double floorLog2 = std::log2(1025.0);
    const double corr = std::fabs(y) > w->gate ? (double)y : 0.0;
    // at most the passing rows (the sample's fraction of the table) and the key range, as estimator.Model
    const double upper = std::min(std::log2(1 + (double)passing * (double)total / (double)std::max<int64_t>(sampled, 1)),
                                  (double)x[4]);
    const double pred =
        std::exp2(std::max(std::min(std::max((double)x[kGroupFeatures - 1], floorLog2) + corr, upper), floorLog2)) - 1;
    cap = std::min(cap, pow2AtLeast(2 * pred * w->margin, 1024));
  }
  return cap;
}

// pre: an aggregator of capacity cap already run for this query (rc: its run's status), as a launch
// shared with other queries leaves it; null: the query's first run happens here.
void serveOne(ws_serve_query& q, const ws_serve_options& o, ws_fetch_status* st, Arena& ar, int64_t cap,
              ws_aggregator* pre = nullptr, int preRc = 0) {
  const int nk = q.plan->nkeys, na = q.plan->naggs;
  const int64_t rowBytes = 8 * (nk + 2 * na);
  const bool arena = !q.keys && !q.accs && !q.exact && o.arena_bytes > 0;
  q.runs = 0;
  q.checksum = 0;
  q.fsum = 0;
  for (;;) {
    ++q.runs;
    ws_aggregator* a = pre;
    int rc = preRc;
    if (pre) {
      pre = nullptr;
    } else {
      checkRc(ws_agg_create(q.plan, cap, nullptr, &a));
      rc = ws_agg_add_batches(a, q.ncols, q.nb, q.bn, q.bdel, q.bcols);
      if (!rc) rc = ws_agg_run(a, q.env, q.jit);
    }
    if (st) {
      // destination: the caller's arrays, or the arena range by range
      const int64_t per = arena ? std::max<int64_t>(1, ar.bytes / rowBytes) : q.max_groups;
      double* dk = arena ? (double*)ar.pinned : q.keys;
      int64_t* dx = arena ? (int64_t*)(ar.pinned + per * 8 * nk) : q.exact;
      int64_t first = 0, groups = 0;
      for (;;) {
        if (!rc) rc = ws_agg_fetch_async(a, first, per, dk, dx, st);
        if (!rc) rc = ws_gpu_sync();
        if (rc) break;
        if (st->error || st->overflow) break;
        groups = st->groups;
        const int64_t got = std::max<int64_t>(0, std::min(per, groups - first));
        if (o.checksum) digest(*q.plan, dk, dx, got, q);
        first += per;
        if (!arena || first >= groups) break;
      }
      ws_agg_destroy(a);
      checkRc(rc);
      if (st->error) throw ws::Error("serve: the aggregation raised an error flag", st->error);
      if (st->overflow) {
        cap = grow(cap, st->groups);
        q.checksum = 0;
        q.fsum = 0;
        continue;
      }
      if (!arena && groups > q.max_groups)
        throw ws::Error("output buffer too small for " + std::to_string(groups) + " groups", WS_ERR_SIZE);
      q.groups = groups;
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
    int64_t g = 0;
    if (arena) {  // the engine's fetch into this worker's host buffer: size query, then the copies
      if (!rc) rc = ws_agg_fetch(a, 0, nullptr, nullptr, nullptr, &g);
      if (rc == WS_ERR_SIZE) rc = 0;
      if (!rc) {
        growTo(ar.host, (size_t)(g * rowBytes));
        double* hk = (double*)ar.host.data();
        int64_t* hx = (int64_t*)(ar.host.data() + g * 8 * nk);
        rc = ws_agg_fetch(a, g, nk ? hk : nullptr, nullptr, hx, &g);
        if (!rc && o.checksum) digest(*q.plan, hk, hx, g, q);
      }
    } else {  // without result arrays or an arena the groups stay on the device (compacted, not downloaded)
      const bool keep = q.keys || q.accs || q.exact;
      if (!rc) rc = ws_agg_fetch(a, keep ? q.max_groups : INT64_MAX, q.keys, q.accs, q.exact, &g);
      if (!rc && keep && o.checksum && q.exact && (q.keys || !nk)) digest(*q.plan, q.keys, q.exact, g, q);
    }
    ws_agg_destroy(a);
    checkRc(rc);
    q.groups = g;
    q.cap_used = cap;
    return;
  }
}

}  // namespace

extern "C" {

int ws_serve(ws_serve_query* queries, int n, const ws_serve_options* opt, double* wall_s) {
  return ws::guardedCall([&] {
    if (!opt) throw ws::Error("serve: options are null", WS_ERR_ARG);
    const ws_serve_options o = *opt;
    if (o.slots < 1 || o.slots > 256) throw ws::Error("serve: 1 to 256 slots", WS_ERR_ARG);
    ws_gpu_init();
    std::mutex mu;
    std::condition_variable cv;
    int64_t inFlight = 0;
    std::atomic<int> next{0}, failed{0};
    std::string firstError;
    int firstCode = 0;
    auto fail = [&](const std::string& m, int code) {
      std::lock_guard<std::mutex> l(mu);
      if (!failed++) firstError = m, firstCode = code;
    };
    // per worker: a stream, the fetch status and the arena (allocated before the clock starts)
    std::vector<cudaStream_t> streams(o.slots, nullptr);
    std::vector<ws_fetch_status*> stat(o.slots, nullptr);
    std::vector<Arena> arenas(o.slots);
    for (int k = 0; k < o.slots && !failed; ++k) {
      if (cudaStreamCreateWithFlags(&streams[k], cudaStreamNonBlocking) != cudaSuccess ||
          (o.one_sync && cudaHostAlloc((void**)&stat[k], sizeof(ws_fetch_status), cudaHostAllocMapped) != cudaSuccess) ||
          (o.one_sync && o.arena_bytes > 0 &&
           cudaHostAlloc((void**)&arenas[k].pinned, (size_t)o.arena_bytes, cudaHostAllocMapped) != cudaSuccess)) {
        cudaGetLastError();
        fail("serve: could not create a worker's stream or pinned buffers", WS_ERR_OOM);
        break;
      }
      arenas[k].bytes = o.one_sync ? o.arena_bytes : 0;
      if (!o.one_sync && o.arena_bytes > 0) {  // touched now, so that the loop does not fault the pages in
        arenas[k].host.resize((size_t)o.arena_bytes);
        std::memset(arenas[k].host.data(), 0, arenas[k].host.size());
      }
    }
    const double t0 = nowS();
    auto worker = [&](int k) {
      ws_set_stream(streams[k]);
      for (;;) {
        const int i = next++;
        if (i >= n || failed) break;
        ws_serve_query& q = queries[i];
        const double wait = q.arrival_s - (nowS() - t0);  // the query has not arrived yet
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        {
          std::unique_lock<std::mutex> l(mu);  // admission by HBM footprint
          cv.wait(l, [&] { return inFlight == 0 || inFlight + q.footprint <= o.hbm_budget; });
          inFlight += q.footprint;
        }
        q.start_s = nowS() - t0;
        // batch: the queries after this one that have arrived, use the same plan (one compiled program,
        // or all interpreted) and fit the budget join its launch (ws_agg_run_many)
        std::vector<int> grp{i};
        while (o.batch > 1 && (int)grp.size() < o.batch && !failed) {
          int j = next.load();
          if (j >= n) break;
          ws_serve_query& c = queries[j];
          if (c.arrival_s > nowS() - t0 || c.jit != q.jit || (c.plan->nkeys == 0) != (q.plan->nkeys == 0)) break;
          std::lock_guard<std::mutex> l(mu);
          if (inFlight + c.footprint > o.hbm_budget) break;
          if (!next.compare_exchange_strong(j, j + 1)) continue;
          inFlight += c.footprint;
          c.start_s = nowS() - t0;
          grp.push_back(j);
        }
        auto oneSyncFor = [&](const ws_serve_query& x) {
          const bool arrays = x.keys || x.accs || x.exact;
          return o.one_sync && (arrays ? (x.keys || !x.plan->nkeys) && x.exact && !x.accs && pinnedHost(x.exact) &&
                                             (!x.keys || pinnedHost(x.keys))
                                       : o.arena_bytes > 0);
        };
        std::vector<ws_aggregator*> pre(grp.size(), nullptr);
        std::vector<int64_t> caps(grp.size(), 0);
        int preRc = 0;
        try {
          if (grp.size() > 1) {  // the first runs of the group in one launch
            std::vector<const ws_expr_env*> envs;
            for (size_t g = 0; g < grp.size(); ++g) {
              ws_serve_query& x = queries[grp[g]];
              caps[g] = initialCap(x, o);
              checkRc(ws_agg_create(x.plan, caps[g], nullptr, &pre[g]));
              checkRc(ws_agg_add_batches(pre[g], x.ncols, x.nb, x.bn, x.bdel, x.bcols));
              envs.push_back(x.env);
            }
            preRc = ws_agg_run_many(pre.data(), envs.data(), q.jit, (int)grp.size());
          } else {
            caps[0] = initialCap(q, o);
          }
        } catch (const ws::Error& e) {
          fail(e.what(), e.code);
          for (auto& a : pre)
            if (a) ws_agg_destroy(a), a = nullptr;
        }
        for (size_t g = 0; g < grp.size(); ++g) {
          ws_serve_query& x = queries[grp[g]];
          ws_aggregator* mine = pre[g];  // serveOne takes it over (and destroys it on every path)
          pre[g] = nullptr;
          try {
            if (failed) {
              if (mine) ws_agg_destroy(mine);
            } else {
              serveOne(x, o, oneSyncFor(x) ? stat[k] : nullptr, arenas[k], caps[g], mine, preRc);
            }
          } catch (const ws::Error& e) {
            fail(e.what(), e.code);
          }
          x.finish_s = nowS() - t0;
          {
            std::lock_guard<std::mutex> l(mu);
            inFlight -= x.footprint;
          }
          cv.notify_all();
        }
      }
      ws_set_stream(nullptr);
    };
    std::vector<std::thread> th;
    if (!failed)
      for (int k = 0; k < o.slots; ++k) th.emplace_back(worker, k);
    for (auto& t : th) t.join();
    if (wall_s) *wall_s = nowS() - t0;
    for (int k = 0; k < o.slots; ++k) {
      if (streams[k]) {
        cudaStreamSynchronize(streams[k]);
        cudaStreamDestroy(streams[k]);
      }
      if (stat[k]) cudaFreeHost(stat[k]);
      if (arenas[k].pinned) cudaFreeHost(arenas[k].pinned);
    }
    if (failed) throw ws::Error(firstError, firstCode ? firstCode : WS_ERR_INTERNAL);
  });
}

}  // extern "C"
