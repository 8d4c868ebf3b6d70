// Host-side internals of libwarpstore_b200: error handling, device runtime, plan analysis and the
// kernel-launch plumbing shared by the operator implementations.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ws_b200.h"
#include "ws_kern.cuh"

namespace ws {

// ---------------------------------------------------------------- errors
// Operators throw Error; the C entry points catch it, record it per thread (ws_last_error) and
// return its code.  Codes follow the engine's SQL error numbers (src/gpu.cu:23-30).
struct Error : std::runtime_error {
  int code;
  Error(const std::string& m, int c = WS_ERR_INTERNAL) : std::runtime_error(m), code(c) {}
};
void setLastError(int code, const std::string& msg);
void ck(cudaError_t e, const char* what);
void ckDrv(CUresult r, const char* what);
#define WS_CK(x) ::ws::ck((x), #x)
#define WS_CKD(x) ::ws::ckDrv((x), #x)

// ---------------------------------------------------------------- runtime
// Driver-API entry points used for loading compiled plans and launching kernels, resolved through the
// runtime (cudaGetDriverEntryPoint) so the library does not link libcuda and loads on hosts without a
// GPU driver (the C ABI is then present; calls report that no device is available).
struct DriverApi {
  CUresult (*moduleLoadData)(CUmodule*, const void*);
  CUresult (*moduleGetFunction)(CUfunction*, CUmodule, const char*);
  CUresult (*launchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                           void**, void**);
  CUresult (*funcSetAttribute)(CUfunction, CUfunction_attribute, int);
  CUresult (*occupancy)(int*, CUfunction, int, size_t);
  CUresult (*getErrorString)(CUresult, const char**);
  CUresult (*graphExecKernelNodeSetParams)(CUgraphExec, CUgraphNode, const CUDA_KERNEL_NODE_PARAMS*);
  CUresult (*funcGetAttribute)(int*, CUfunction_attribute, CUfunction);
};
const DriverApi& drv();
void ensureInit();
int smCount();
int arch();
cudaStream_t stream();           // the calling thread's stream (ws_set_stream), default per-thread
void* tmpAlloc(size_t bytes);    // stream-ordered pool allocation on stream()
void tmpFree(void* p);
void h2dAsync(void* d, const void* h, size_t b);
void d2hSync(void* h, const void* d, size_t b);
// The same for large copies into pageable memory: pipelined through pinned staging (synchronous).
void d2hLarge(void* h, const void* d, size_t b);
void sync();
void countLaunch(int n = 1);     // kernels launched by this library (ws_kernel_launches)
// Launch-shape autotuner (ws_tune.cpp): a scan's CTAs per SM (0: as many as fit) and, for the hash
// scan, the per-CTA table's shared-memory budget in KB (0: the default).
struct TuneChoice {
  int ctasPerSm = 0;
  int smemKB = 0;
  int stages = -1;  // shared-memory tile stages of a compiled scan (0: direct loads; -1: the default)
  int slotsPerKey = 0;  // a hash join's table slots per build key (0: the default)
  bool found = false;
};
int tuneMode();  // WS_TUNE_USE / WS_TUNE_ON / WS_TUNE_OFF
std::string tuneKey(const char* kernel, const ws_jit_program* jit, const ws_agg_plan& plan, int64_t ntiles);
bool tuneLookup(const std::string& key, TuneChoice& c);
void tuneStore(const std::string& key, const TuneChoice& c, double us);
void tuneSetDir(const std::string& dir);  // "" : memory only
void setStream(cudaStream_t s);
// Runs f, translating exceptions into the calling thread's last error; returns the error code.
int guardedCall(const std::function<void()>& f);

// RAII stream-ordered device buffer
template <class T>
struct DBuf {
  T* p = nullptr;
  int64_t n = 0;
  DBuf() = default;
  explicit DBuf(int64_t count) : n(count) { p = count > 0 ? (T*)tmpAlloc(sizeof(T) * count) : nullptr; }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr, o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p, n = o.n;
      o.p = nullptr, o.n = 0;
    }
    return *this;
  }
  ~DBuf() { reset(); }
  void reset() {
    if (p) tmpFree(p);
    p = nullptr, n = 0;
  }
  T* release() {
    T* q = p;
    p = nullptr, n = 0;
    return q;
  }
};

// Pinned staging for small host <-> device descriptor copies (per thread, reused once the previous
// copy out of it has completed).
uint8_t* pinnedStage(size_t bytes);
void stageCopied();  // records that the copy out of the staging buffer has been issued

// ---------------------------------------------------------------- plan analysis
// A node of an expression tree rebuilt from the engine's stack bytecode, typed as the code generator
// types it: integer columns / literals / arithmetic stay int64, everything else is double.
struct TNode {
  uint8_t op = 0, instrInt = 0;
  uint16_t arg = 0;
  bool isInt = false;
  int kid[3] = {-1, -1, -1};
};
struct TypedProg {
  std::vector<TNode> nodes;
  int root = -1;
  bool isInt() const { return nodes[root].isInt; }
};
TypedProg typeProg(const ws_expr_env& env, ws_prog p, int ncols);

// Accumulator row layout of a plan: word 0 = key word, slot a at woff[a] (0 .. 2 words).
struct SlotLayout {
  int na = 0, rw = 1;
  uint8_t kind[WS_MAX_AGGS] = {};
  int woff[WS_MAX_AGGS] = {};
  int partner[WS_MAX_AGGS] = {};  // SK_NONE slots: the slot whose value they repeat
  int fwoff[WS_MAX_AGGS] = {};    // word of the slot in per-thread register rows
  int frw = 0;                    // words of a register row
};
SlotLayout layoutOf(const ws_agg_plan& plan);
// Typed interpreter code for the plan's programs (where, keys, aggregates).
void buildTProgs(const ws_expr_env& env, int ncols, const ws_agg_plan& plan, bool hasWhere, TProgs& out);
EnvK envK(const ws_expr_env& env);

// ---------------------------------------------------------------- kernels
// The scan kernels of one evaluator: the interpreter's (built into the library) or a compiled plan's.
// K_DENSE_PRIV: direct loads, kThreads threads, bounded for several resident CTAs per SM;
// K_DENSE_PRIV_STAGED: the same body with a producer warp staging tiles by TMA (kStagedThreads).
enum KernelId {
  K_NOKEYS = 0, K_DENSE_SHARED, K_DENSE_GLOBAL, K_HASH, K_SELECT_COUNT, K_SELECT_WRITE, K_DENSE_PRIV,
  K_DENSE_PRIV_STAGED, K_MULTI_NOKEYS, K_MULTI_DENSE_PRIV, K_MULTI_HASH, K_COUNT_
};
struct KernelSet {
  CUfunction fn[K_COUNT_] = {};
  bool interp = true;
};
const KernelSet& interpKernels();
// Raises f's dynamic shared memory allowance to smem (never lowers it; safe across threads).
void allowDynamicSmem(CUfunction f, size_t smem);
// Launch.sumShift of a scan of ntiles tiles on `grid` CTAs (the integer SUM bound of ws_kern.cuh).
int sumShiftFor(int64_t ntiles, unsigned grid);
// Launch.waitLog2: the staged scans' wait limit (WARPSTORE_B200_WAIT_LIMIT_LOG2, default 32).
int stagedWaitLog2();
// Launches `f` with the Launch descriptor as its only parameter (sumShift set for the grid).
void launchScan(CUfunction f, unsigned grid, size_t smem, const Launch& L, int threads = kThreads);
// Persistent grid: resident CTAs per SM x SMs, capped by the tile count.
unsigned persistentGrid(CUfunction f, size_t smem, int64_t ntiles, int threads = kThreads);

}  // namespace ws

// A compiled plan (the engine's JitProgram, src/jit.h:16-31): generated evaluator source, its module
// and kernels, state and statistics.
struct ws_jit_program {
  int id = 0;
  int fnKind = 0;
  std::string kind, sql, source;
  double compileMs = 0;
  std::atomic<int> state{0};  // 0 compiling, 1 ready, 2 failed
  bool fromDisk = false;
  int stageBytes = 0;  // shared memory per staged tile (0: the plan reads global memory directly)
  ws::KernelSet kernels;
  CUmodule module = nullptr;
  std::mutex mu;
  int64_t execs = 0;
  double totalMs = 0, lastMs = 0;
};

