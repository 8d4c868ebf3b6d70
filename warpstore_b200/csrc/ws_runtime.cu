// Device runtime of libwarpstore_b200: initialisation, per-thread streams, the stream-ordered memory
// pool, pinned staging, error reporting and the launch helpers (reference: src/gpu.cu:23-240).
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <thread>

#include "ws_internal.h"

namespace ws {

namespace {
thread_local int tErrCode = 0;
thread_local std::string tErrMsg;
thread_local cudaStream_t tStream = nullptr;
thread_local bool tStreamSet = false;
std::once_flag gInitOnce;
int gSms = 148, gArch = 100;
std::atomic<int64_t> gLaunches{0};
}  // namespace

void setLastError(int code, const std::string& msg) {
  tErrCode = code;
  tErrMsg = msg;
}

void ck(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    throw Error("GPU out of memory", WS_ERR_OOM);
  }
  throw Error(std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + what, WS_ERR_INTERNAL);
}

void ckDrv(CUresult r, const char* what) {
  if (r == CUDA_SUCCESS) return;
  const char* msg = nullptr;
  if (drv().getErrorString) drv().getErrorString(r, &msg);
  if (r == CUDA_ERROR_OUT_OF_MEMORY) throw Error("GPU out of memory", WS_ERR_OOM);
  throw Error(std::string("CUDA driver error: ") + (msg ? msg : "?") + " at " + what, WS_ERR_INTERNAL);
}

void ensureInit() {
  std::call_once(gInitOnce, [] {
    int dev = 0;
    WS_CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    WS_CK(cudaGetDeviceProperties(&prop, dev));
    gSms = prop.multiProcessorCount;
    gArch = prop.major * 10 + prop.minor;
    // Query temporaries come from the stream-ordered pool, which keeps freed memory for the next
    // queries instead of returning it at every synchronization.
    cudaMemPool_t pool;
    WS_CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thresh = UINT64_MAX;
    WS_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
    (void)drv();
  });
}

const DriverApi& drv() {
  static DriverApi api = [] {
    DriverApi a{};
    auto get = [](const char* name, void** fn) {
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        throw Error(std::string("CUDA driver entry point unavailable: ") + name, WS_ERR_INTERNAL);
      }
    };
    get("cuModuleLoadData", (void**)&a.moduleLoadData);
    get("cuModuleGetFunction", (void**)&a.moduleGetFunction);
    get("cuLaunchKernel", (void**)&a.launchKernel);
    get("cuFuncSetAttribute", (void**)&a.funcSetAttribute);
    get("cuOccupancyMaxActiveBlocksPerMultiprocessor", (void**)&a.occupancy);
    get("cuGetErrorString", (void**)&a.getErrorString);
    get("cuGraphExecKernelNodeSetParams", (void**)&a.graphExecKernelNodeSetParams);
    get("cuFuncGetAttribute", (void**)&a.funcGetAttribute);
    return a;
  }();
  return api;
}

int smCount() {
  ensureInit();
  return gSms;
}
int arch() {
  ensureInit();
  return gArch;
}

cudaStream_t stream() { return tStreamSet ? tStream : cudaStreamPerThread; }
void setStream(cudaStream_t s) {
  tStream = s;
  tStreamSet = s != nullptr;
}

static void trimPool() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
  cudaDeviceSynchronize();
  cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
}

void* tmpAlloc(size_t bytes) {
  if (!bytes) return nullptr;
  ensureInit();
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, stream()) != cudaSuccess) {  // once more with the pool's spare memory released
    cudaGetLastError();
    trimPool();
    WS_CK(cudaMallocAsync(&p, bytes, stream()));
  }
  return p;
}
void tmpFree(void* p) {
  if (p) cudaFreeAsync(p, stream());
}
void h2dAsync(void* d, const void* h, size_t b) {
  if (b) WS_CK(cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, stream()));
}
void d2hSync(void* h, const void* d, size_t b) {
  if (!b) return;
  WS_CK(cudaMemcpyAsync(h, d, b, cudaMemcpyDeviceToHost, stream()));
  WS_CK(cudaStreamSynchronize(stream()));
}
void sync() { WS_CK(cudaStreamSynchronize(stream())); }
void countLaunch(int n) { gLaunches += n; }

// ---- large device -> pageable host copies
// A copy into pageable memory runs at a fraction of the link speed (the driver stages it and the
// destination pages fault in on one thread).  Large copies go through a per-thread pinned ring
// instead: chunk i is copied by DMA into a ring slot while chunks already landed are copied out of
// their slots by a small pool of host threads.
namespace {
constexpr size_t kRingChunk = 8u << 20;
constexpr int kRingSlots = 4;
struct PinnedRing {
  uint8_t* buf = nullptr;
  cudaEvent_t ev[kRingSlots] = {};
};
thread_local PinnedRing tRing;

class CopyPool {
 public:
  explicit CopyPool(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
  }
  int size() const { return (int)th_.size(); }
  // memcpy of n bytes split across the pool and the calling thread; returns when all parts are done
  void copy(uint8_t* dst, const uint8_t* src, size_t n) {
    const int parts = size() + 1;
    const size_t per = (n + parts - 1) / parts;
    std::atomic<int> left{0};
    {
      std::lock_guard<std::mutex> l(mu_);
      for (int p = 1; p < parts; ++p) {
        const size_t lo = std::min(n, per * p), hi = std::min(n, lo + per);
        if (hi > lo) {
          ++left;
          q_.push_back({dst + lo, src + lo, hi - lo, &left});
        }
      }
    }
    cv_.notify_all();
    memcpy(dst, src, std::min(n, per));
    std::unique_lock<std::mutex> l(mu_);
    done_.wait(l, [&] { return left.load() == 0; });
  }

 private:
  struct Job {
    uint8_t* dst;
    const uint8_t* src;
    size_t n;
    std::atomic<int>* left;
  };
  void loop() {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return !q_.empty(); });
        j = q_.front();
        q_.pop_front();
      }
      memcpy(j.dst, j.src, j.n);
      std::lock_guard<std::mutex> l(mu_);
      if (--*j.left == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::deque<Job> q_;
};
CopyPool& copyPool() {  // process-wide; never destroyed (its threads idle until exit)
  static CopyPool* p = new CopyPool((int)std::max(1u, std::min(7u, std::thread::hardware_concurrency() / 2)));
  return *p;
}
}  // namespace

void d2hLarge(void* h, const void* d, size_t b) {
  if (b < 2 * kRingChunk) {
    d2hSync(h, d, b);
    return;
  }
  PinnedRing& r = tRing;
  if (!r.buf) {
    WS_CK(cudaHostAlloc((void**)&r.buf, kRingChunk * kRingSlots, cudaHostAllocDefault));
    for (auto& e : r.ev) WS_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const size_t nchunks = (b + kRingChunk - 1) / kRingChunk;
  auto issue = [&](size_t i) {
    const int slot = (int)(i % kRingSlots);
    const size_t lo = i * kRingChunk, n = std::min(kRingChunk, b - lo);
    WS_CK(cudaMemcpyAsync(r.buf + (size_t)slot * kRingChunk, (const uint8_t*)d + lo, n, cudaMemcpyDeviceToHost, stream()));
    WS_CK(cudaEventRecord(r.ev[slot], stream()));
  };
  for (size_t i = 0; i < std::min<size_t>(kRingSlots, nchunks); ++i) issue(i);
  for (size_t i = 0; i < nchunks; ++i) {
    const int slot = (int)(i % kRingSlots);
    WS_CK(cudaEventSynchronize(r.ev[slot]));
    const size_t lo = i * kRingChunk, n = std::min(kRingChunk, b - lo);
    copyPool().copy((uint8_t*)h + lo, r.buf + (size_t)slot * kRingChunk, n);
    if (i + kRingSlots < nchunks) issue(i + kRingSlots);
  }
}

// Per-thread pinned staging buffer; an event marks the last copy out of it so reuse waits only then.
namespace {
thread_local uint8_t* tStage = nullptr;
thread_local size_t tStageCap = 0;
thread_local cudaEvent_t tStageEv = nullptr;
}  // namespace
uint8_t* pinnedStage(size_t bytes) {
  if (tStageEv) WS_CK(cudaEventSynchronize(tStageEv));
  else WS_CK(cudaEventCreateWithFlags(&tStageEv, cudaEventDisableTiming));
  if (bytes > tStageCap) {
    if (tStage) cudaFreeHost(tStage);
    tStageCap = std::max<size_t>(bytes, 64 << 10);
    WS_CK(cudaHostAlloc((void**)&tStage, tStageCap, cudaHostAllocDefault));
  }
  return tStage;
}
void stageCopied() { WS_CK(cudaEventRecord(tStageEv, stream())); }

int stagedWaitLog2() {
  // WARPSTORE_B200_WAIT_LIMIT_LOG2 (4..32, default 32 = ~2 s): how long a staged scan waits for a tile
  // stage before it reports the tile as late (err[2]); a small value makes the waits run out (tests)
  static const int v = [] {
    const char* e = getenv("WARPSTORE_B200_WAIT_LIMIT_LOG2");
    const int x = e ? atoi(e) : 32;
    return x < 4 ? 4 : x > 32 ? 32 : x;
  }();
  return v;
}

int sumShiftFor(int64_t ntiles, unsigned grid) {
  // rows one thread adds into a word: 4 per tile, ceil(ntiles / grid) tiles per CTA (contiguous ranges)
  const int64_t g = grid ? grid : 1;
  const int64_t rows = std::max<int64_t>(1, (ntiles + g - 1) / g) * 4;
  int k = 0;
  while (((int64_t)1 << k) < rows) ++k;
  return k <= 31 ? 31 - k : -1;
}

void allowDynamicSmem(CUfunction f, size_t smem) {
  // The attribute is per function and shared by every thread that launches it: it only ever grows
  // (under a lock), so that a thread asking for less never lowers it below another thread's launch.
  if (!smem) return;
  static std::mutex mu;
  static std::map<CUfunction, size_t> allowed;
  std::lock_guard<std::mutex> g(mu);
  size_t& cur = allowed[f];
  if (smem <= cur) return;
  WS_CKD(drv().funcSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem));
  cur = smem;
}

void launchScan(CUfunction f, unsigned grid, size_t smem, const Launch& Lin, int threads) {
  allowDynamicSmem(f, smem);
  Launch L = Lin;
  L.sumShift = sumShiftFor(L.ntiles, grid);
  L.waitLog2 = stagedWaitLog2();
  void* args[] = {(void*)&L};
  WS_CKD(drv().launchKernel(f, grid, 1, 1, (unsigned)threads, 1, 1, (unsigned)smem, (CUstream)stream(), args, nullptr));
  countLaunch();
}

unsigned persistentGrid(CUfunction f, size_t smem, int64_t ntiles, int threads) {
  allowDynamicSmem(f, smem);
  int per = 0;
  WS_CKD(drv().occupancy(&per, f, threads, smem));
  if (per < 1) {
    int regs = 0, stat = 0, local = 0, maxThreads = 0;
    drv().funcGetAttribute(&regs, CU_FUNC_ATTRIBUTE_NUM_REGS, f);
    drv().funcGetAttribute(&stat, CU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES, f);
    drv().funcGetAttribute(&local, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, f);
    drv().funcGetAttribute(&maxThreads, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, f);
    throw Error("scan kernel does not fit on an SM (" + std::to_string(threads) + " threads, dynamic shared memory " +
                    std::to_string(smem) + " B, static " + std::to_string(stat) + " B, " + std::to_string(regs) +
                    " registers, local " + std::to_string(local) + " B, at most " + std::to_string(maxThreads) +
                    " threads)",
                WS_ERR_INTERNAL);
  }
  int64_t g = (int64_t)per * smCount();
  if (g > ntiles) g = ntiles;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace ws

using namespace ws;

// Runs f, translating exceptions into the thread's last error.
template <class F>
static int guarded(F&& f) {
  try {
    f();
    return WS_OK;
  } catch (const Error& e) {
    setLastError(e.code, e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    setLastError(WS_ERR_OOM, "host out of memory");
    return WS_ERR_OOM;
  } catch (const std::exception& e) {
    setLastError(WS_ERR_INTERNAL, e.what());
    return WS_ERR_INTERNAL;
  }
}

extern "C" {

const char* ws_last_error(void) { return tErrMsg.c_str(); }
int ws_last_error_code(void) { return tErrCode; }

int ws_gpu_init(void) { return guarded([] { ensureInit(); }); }
int ws_gpu_sm_count(void) {
  int r = 0;
  guarded([&] { r = smCount(); });
  return r;
}
int ws_gpu_arch(void) {
  int r = 0;
  guarded([&] { r = arch(); });
  return r;
}
int ws_gpu_describe(char* buf, size_t size) {
  return guarded([&] {
    ensureInit();
    int dev = 0;
    WS_CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    WS_CK(cudaGetDeviceProperties(&prop, dev));
    size_t fr = 0, tot = 0;
    WS_CK(cudaMemGetInfo(&fr, &tot));
    snprintf(buf, size, "%s (sm_%d%d, %d SMs, %.1f GiB free / %.1f GiB)", prop.name, prop.major, prop.minor,
             prop.multiProcessorCount, fr / 1073741824.0, tot / 1073741824.0);
  });
}
int ws_set_stream(void* s) {
  setStream((cudaStream_t)s);
  return WS_OK;
}
void* ws_get_stream(void) { return (void*)stream(); }
int ws_dev_alloc(size_t bytes, void** out) {
  return guarded([&] {
    ensureInit();
    *out = nullptr;
    if (bytes) WS_CK(cudaMalloc(out, bytes));
  });
}
int ws_dev_free(void* p) {
  return guarded([&] {
    if (p) WS_CK(cudaFree(p));
  });
}
int ws_tmp_alloc(size_t bytes, void** out) { return guarded([&] { *out = tmpAlloc(bytes); }); }
int ws_tmp_free(void* p) { return guarded([&] { tmpFree(p); }); }
int ws_h2d(void* dst, const void* src, size_t bytes) {
  return guarded([&] {
    if (bytes) {
      WS_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream()));
      WS_CK(cudaStreamSynchronize(stream()));
    }
  });
}
int ws_d2h(void* dst, const void* src, size_t bytes) { return guarded([&] { d2hLarge(dst, src, bytes); }); }
int ws_d2d(void* dst, const void* src, size_t bytes) {
  return guarded([&] {
    if (bytes) WS_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream()));
  });
}
int ws_gpu_sync(void) { return guarded([] { sync(); }); }
int ws_gpu_trim_pool(void) { return guarded([] { trimPool(); }); }

int ws_abi_layout(int64_t* out, int n) {
  const int64_t v[] = {(int64_t)sizeof(ws_instr),
                       (int64_t)sizeof(ws_col_view),
                       (int64_t)offsetof(ws_col_view, off),
                       (int64_t)sizeof(ws_expr_env),
                       (int64_t)offsetof(ws_expr_env, consts),
                       (int64_t)offsetof(ws_expr_env, sets),
                       (int64_t)offsetof(ws_expr_env, setSize),
                       (int64_t)offsetof(ws_expr_env, maps),
                       (int64_t)offsetof(ws_expr_env, mapSize),
                       (int64_t)offsetof(ws_expr_env, cols),
                       (int64_t)offsetof(ws_expr_env, ovf),
                       (int64_t)sizeof(ws_agg_plan),
                       (int64_t)offsetof(ws_agg_plan, where),
                       (int64_t)offsetof(ws_agg_plan, nkeys),
                       (int64_t)offsetof(ws_agg_plan, keys),
                       (int64_t)offsetof(ws_agg_plan, naggs),
                       (int64_t)offsetof(ws_agg_plan, aggs),
                       (int64_t)offsetof(ws_agg_plan, ops),
                       (int64_t)offsetof(ws_agg_plan, aggInt),
                       (int64_t)offsetof(ws_agg_plan, aggBits),
                       (int64_t)offsetof(ws_agg_plan, aggPart),
                       (int64_t)offsetof(ws_agg_plan, aggNull),
                       (int64_t)offsetof(ws_agg_plan, densePriv),
                       (int64_t)offsetof(ws_agg_plan, keyInt),
                       (int64_t)offsetof(ws_agg_plan, genv),
                       (int64_t)sizeof(ws_dense_spec),
                       (int64_t)offsetof(ws_dense_spec, kmin),
                       (int64_t)offsetof(ws_dense_spec, range),
                       (int64_t)offsetof(ws_dense_spec, stride),
                       (int64_t)offsetof(ws_dense_spec, slotOff),
                       (int64_t)offsetof(ws_dense_spec, kind)};
  const int m = (int)(sizeof v / sizeof v[0]);
  for (int i = 0; i < n && i < m; ++i) out[i] = v[i];
  return m;
}

int64_t ws_kernel_launches(void) { return gLaunches.load(); }

}  // extern "C"

namespace ws {
int guardedCall(const std::function<void()>& f) { return guarded(f); }
}  // namespace ws
