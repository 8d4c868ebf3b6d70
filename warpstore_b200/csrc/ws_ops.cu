// Operators of libwarpstore_b200: aggregation (GpuAggregator), selection, gathers and hash joins
// (reference: src/gpu.cu:393-800, :1089-1316).  Scan kernels come from ws_kern.cuh, instantiated here
// with the interpreter and per plan by the code generator; the helper kernels below are plain CUDA.
#include <cstring>

#include "ws_internal.h"

namespace ws {

// Interpreter instantiations of every scan kernel (prefix wsi), one translation unit per group.
void interpSyms_agg(const void** s);
void interpSyms_priv(const void** s);
void interpSyms_hash(const void** s);
void interpSyms_select(const void** s);

const KernelSet& interpKernels() {
  static KernelSet ks = [] {
    KernelSet k;
    const void* syms[K_COUNT_] = {};
    interpSyms_agg(syms);
    interpSyms_priv(syms);
    interpSyms_hash(syms);
    interpSyms_select(syms);
    for (int i = 0; i < K_COUNT_; ++i) {
      cudaFunction_t f;
      WS_CK(cudaGetFuncBySymbol(&f, syms[i]));
      k.fn[i] = (CUfunction)f;
    }
    k.interp = true;
    return k;
  }();
  return ks;
}

namespace {

int gridFor(int64_t n, int block = 256, int perSm = 8) {
  int64_t g = (n + block - 1) / block;
  const int64_t cap = (int64_t)smCount() * perSm;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}
#define WS_LAUNCH(kernel, grid, block, smem, ...)                 \
  do {                                                            \
    kernel<<<(grid), (block), (smem), stream()>>>(__VA_ARGS__);   \
    WS_CK(cudaGetLastError());                                    \
    countLaunch();                                                \
  } while (0)

// ---------------------------------------------------------------- helper kernels
}  // namespace
// Identity values of one accumulator row (by value as a kernel parameter).
struct RowTemplate {
  u64 w[kMaxRowWords];
};
namespace {
__global__ void kFillRows(u64* rows, int64_t nrows, int rw, RowTemplate t, int64_t emptyRows) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
    u64* r = rows + i * rw;
    for (int j = 1; j < rw; ++j) r[j] = t.w[j];
    r[0] = i < emptyRows ? kEmpty : 0ull;
  }
}

// Exclusive scan of n counts in place (one CTA); counts[n] receives the total.
__global__ void kScanExclusive(int64_t* counts, int64_t n) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int64_t per = (n + T - 1) / T;
  const int64_t lo = min((int64_t)t * per, n), hi = min(lo + per, n);
  int64_t s = 0;
  for (int64_t i = lo; i < hi; ++i) s += counts[i];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {  // Hillis-Steele inclusive scan of the thread sums
    const int64_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = t ? part[t - 1] : 0;
  for (int64_t i = lo; i < hi; ++i) {
    const int64_t c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (t == T - 1) counts[n] = part[T - 1];
}

// Occupied result rows: hash rows [0, cap) by their key word, the extra row (cap) by its claim flag,
// dense rows by slot 0 (COUNT(*)) being non-zero.
struct OccSpec {
  int rw, mode;  // mode 1 dense, 2 hash
  int cnt0;      // word of slot 0
  int64_t cap;   // hash: index of the extra row
};
__device__ __forceinline__ bool occupied(const u64* rows, int64_t i, const OccSpec& s) {
  const u64* r = rows + i * s.rw;
  if (s.mode == 0) return true;  // no GROUP BY: the one result row
  if (s.mode == 1) return r[s.cnt0] != 0;
  if (i == s.cap) return r[0] != 0;
  return r[0] != kEmpty;
}
constexpr int kOccChunk = 2048;
__global__ void kOccCount(const u64* rows, int64_t nrows, OccSpec s, int64_t* counts) {
  __shared__ int wc[32];
  const int64_t c0 = (int64_t)blockIdx.x * kOccChunk;
  int c = 0;
  for (int64_t i = c0 + threadIdx.x; i < min(c0 + kOccChunk, nrows); i += blockDim.x) c += occupied(rows, i, s);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wc[w];
    counts[blockIdx.x] = t;
  }
}
__global__ void kOccWrite(const u64* rows, int64_t nrows, OccSpec s, const int64_t* offs, int64_t* idx) {
  __shared__ int wbase[32];
  __shared__ int64_t run;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t c0 = (int64_t)blockIdx.x * kOccChunk;
  if (threadIdx.x == 0) run = offs[blockIdx.x];
  __syncthreads();
  for (int64_t b = c0; b < min(c0 + kOccChunk, nrows); b += blockDim.x) {
    const int64_t i = b + threadIdx.x;
    const bool occ = i < nrows && i < c0 + kOccChunk && occupied(rows, i, s);
    const unsigned m = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) wbase[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) before += wbase[w];
      total += wbase[w];
    }
    if (occ) idx[run + before + __popc(m & ((1u << lane) - 1))] = i;
    __syncthreads();
    if (threadIdx.x == 0) run += total;
    __syncthreads();
  }
}

// Result rows -> keys (engine format) and exact words per group.
struct EmitSpec {
  int nk, na, rw, mode;  // mode 0 no keys, 1 dense, 2 hash
  uint8_t kind[WS_MAX_AGGS];
  int16_t woff[WS_MAX_AGGS];
  int16_t partner[WS_MAX_AGGS];
  uint8_t keyInt[WS_MAX_KEYS];
  int64_t kmin[WS_MAX_KEYS], range[WS_MAX_KEYS], stride[WS_MAX_KEYS];
  const double* tkeys;
  int64_t cap;
};
// Keys (engine format) and exact words of result row i: key k at kout[k * kstride], slot a at
// xout[2a], xout[2a + 1].
__device__ __forceinline__ void emitRow(const u64* rows, int64_t i, const EmitSpec& s, double* kout, int64_t kstride,
                                        long long* xout) {
  const u64* r = rows + i * s.rw;
  for (int k = 0; k < s.nk; ++k) {
    double kv;
    if (s.mode == 1) {
      const long long v = s.kmin[k] + (i / s.stride[k]) % s.range[k];
      kv = s.keyInt[k] ? __longlong_as_double(v) : (double)v;
    } else if (s.nk == 1 && i != s.cap) {
      kv = __longlong_as_double((long long)r[0]);
    } else {
      kv = s.tkeys[i * s.nk + k];
    }
    kout[k * kstride] = kv;
  }
  for (int a = 0; a < s.na; ++a) {
    const int src = s.kind[a] == SK_NONE ? s.partner[a] : a;
    const int o = s.woff[src];
    long long w0 = (long long)r[o], w1 = 0;
    const uint8_t k = s.kind[src];
    if (k == SK_ISUM) w1 = (long long)r[o + 1];
    else if (k == SK_DMIN || k == SK_DMAX) w0 = __double_as_longlong(dunord(w0));
    xout[2 * a] = w0;
    xout[2 * a + 1] = w1;
  }
}

__global__ void kEmit(const u64* rows, const int64_t* idx, int64_t m, EmitSpec s, double* keys, int64_t* exact,
                      int colMajor) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx ? idx[j] : j;
    emitRow(rows, i, s, colMajor ? keys + j : keys + j * s.nk, colMajor ? m : 1, (long long*)exact + j * s.na * 2);
  }
}

// Fetch straight into host memory (pinned and mapped): group p (ascending result-row order; the groups
// of chunk b of kOccChunk result rows are offs[b]..) goes to output row p - first when first <= p <
// first + limit.  One sub-tile of blockDim result rows at a time, its rows staged in shared memory
// ([blockDim][nk + 2 na] words) and stored as contiguous words (whole PCIe writes rather than one
// 8-byte write per word of a row).  Nothing is written when the run raised a flag (hash overflow, dense
// key out of range, staged-copy timeout): the caller reads the status and reruns.
__global__ void kOccEmitHost(const u64* rows, int64_t nrows, OccSpec o, EmitSpec s, const int64_t* offs, int64_t nchunks,
                             const int* err, int64_t first, int64_t limit, double* keys, long long* exact) {
  extern __shared__ long long stg[];
  __shared__ int wbase[32];
  if (err[0] || err[2] || (o.mode == 2 && err[1])) return;
  if (offs[blockIdx.x + 1] <= first || offs[blockIdx.x] >= first + limit) return;  // none of this chunk's groups
  const int64_t last = first + limit;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int xw = 2 * s.na, rw = s.nk + xw;
  const int64_t c0 = (int64_t)blockIdx.x * kOccChunk, cend = min(c0 + kOccChunk, nrows);
  int64_t run = offs[blockIdx.x];
  for (int64_t b = c0; b < cend; b += blockDim.x) {
    const int64_t i = b + threadIdx.x;
    const bool occ = i < cend && occupied(rows, i, o);
    const unsigned m = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) wbase[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) before += wbase[w];
      total += wbase[w];
    }
    if (occ) {
      long long* r = stg + (int64_t)(before + __popc(m & ((1u << lane) - 1))) * rw;
      emitRow(rows, i, s, (double*)r, 1, r + s.nk);
    }
    __syncthreads();
    // this sub-tile's groups [run, run + total) clipped to [first, last), at output row p - first
    const int lo = (int)min((int64_t)total, max((int64_t)0, first - run));
    const int hi = (int)max((int64_t)lo, min((int64_t)total, last - run));
    for (int t = lo * s.nk + threadIdx.x; t < hi * s.nk; t += blockDim.x)
      keys[(run - first) * s.nk + t] = __longlong_as_double(stg[(t / s.nk) * rw + t % s.nk]);
    for (int t = lo * xw + threadIdx.x; t < hi * xw; t += blockDim.x)
      exact[(run - first) * xw + t] = stg[(t / xw) * rw + s.nk + t % xw];
    run += total;
    __syncthreads();
  }
}

// Status of an asynchronous fetch, in host memory (pinned and mapped).
__global__ void kFetchStatus(const int64_t* total, const int* err, int hashMode, ws_fetch_status* st) {
  st->groups = *total;
  st->overflow = hashMode && err[1] ? 1 : 0;
  st->error = err[0] ? WS_ERR_RANGE : err[2] ? WS_ERR_INTERNAL : 0;
}

// Exact words -> the engine's double slot format, on the device (for compact()).
struct DblSpec {
  int na, nokeys;
  uint8_t kind[WS_MAX_AGGS], aggBits[WS_MAX_AGGS], aggPart[WS_MAX_AGGS];
};
__device__ __host__ inline double bitsToD(long long v) {
  double d;
  memcpy(&d, &v, 8);
  return d;
}
__device__ __host__ inline double slotDouble(const DblSpec& s, int a, long long w0, long long w1, bool srcIsNone,
                                             uint8_t srcKind) {
  const uint8_t k = srcKind;
  if (k == SK_COUNT) return (double)w0;
  if (k == SK_ISUM) {
    const __int128 T = (__int128)(((unsigned __int128)(unsigned long long)w1 << 64) | (unsigned long long)w0);
    if (s.nokeys) {
      long long lo = w0;
      double d;
      memcpy(&d, &lo, 8);
      return d;
    }
    if (s.aggBits[a]) {
      long long v = s.aggPart[a] == 2 || srcIsNone ? (long long)(T >> 32) : s.aggPart[a] == 1 ? (long long)(T & 0xffffffff) : w0;
      double d;
      memcpy(&d, &v, 8);
      return d;
    }
    return (double)T;
  }
  if (k == SK_IMIN || k == SK_IMAX) {
    if (s.nokeys || s.aggBits[a]) {
      double d;
      memcpy(&d, &w0, 8);
      return d;
    }
    if (k == SK_IMIN && w0 == 0x7fffffffffffffffll) return bitsToD(0x7ff0000000000000ll);
    if (k == SK_IMAX && w0 == (long long)0x8000000000000000ull) return bitsToD((long long)0xfff0000000000000ull);
    return (double)w0;
  }
  double d;
  memcpy(&d, &w0, 8);
  return d;
}
// colMajor: accs[a * m + j] (compact) else accs[j * na + a] (fetch)
__global__ void kExactToDouble(const int64_t* exact, int64_t m, DblSpec s, const int16_t* partnerKinds, double* accs,
                               int colMajor) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x)
    for (int a = 0; a < s.na; ++a) {
      const bool none = s.kind[a] == SK_NONE;
      const uint8_t sk = none ? (uint8_t)partnerKinds[a] : s.kind[a];
      accs[colMajor ? a * m + j : j * s.na + a] =
          slotDouble(s, a, exact[(j * s.na + a) * 2], exact[(j * s.na + a) * 2 + 1], none, sk);
    }
}

}  // namespace

// ---------------------------------------------------------------- batch descriptor
// Device copy of the batches of one launch: [cols nb*ncols][n nb][del nb][tileStart nb+1][rowStart nb+1]
// followed, for interpreted plans, by the typed programs and slot tables.
struct BatchDesc {
  DBuf<uint8_t> buf;
  int64_t ntiles = 0, rows = 0;
  const ws_col_view* cols = nullptr;
  const int64_t* n = nullptr;
  const uint32_t* const* del = nullptr;
  const int64_t* tileStart = nullptr;
  const int64_t* rowStart = nullptr;
  const TProgs* progs = nullptr;
  const uint8_t* kinds = nullptr;
  const int* woff = nullptr;
  const int* fwoff = nullptr;
  const uint8_t* aggNull = nullptr;
  const uint8_t* keyInt = nullptr;
};

static BatchDesc uploadBatches(int nb, int ncols, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                               const TProgs* progs, const SlotLayout* lay, const ws_agg_plan* plan) {
  BatchDesc d;
  const size_t colBytes = (size_t)nb * ncols * sizeof(ws_col_view);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = (off + 15) & ~(size_t)15;
    off = o + bytes;
    return o;
  };
  const size_t oCols = take(colBytes), oN = take(8 * nb), oDel = take(8 * nb), oTile = take(8 * (nb + 1)),
               oRow = take(8 * (nb + 1));
  size_t oProg = 0, oKinds = 0, oWoff = 0, oFwoff = 0, oNull = 0, oKeyInt = 0;
  if (progs) {
    oProg = take(sizeof(TProgs));
    oKinds = take(WS_MAX_AGGS);
    oWoff = take(4 * WS_MAX_AGGS);
    oFwoff = take(4 * WS_MAX_AGGS);
    oNull = take(WS_MAX_AGGS);
    oKeyInt = take(WS_MAX_KEYS);
  }
  uint8_t* st = pinnedStage(off);
  memcpy(st + oCols, bcols, colBytes);
  int64_t* n = (int64_t*)(st + oN);
  const uint32_t** del = (const uint32_t**)(st + oDel);
  int64_t* ts = (int64_t*)(st + oTile);
  int64_t* rs = (int64_t*)(st + oRow);
  ts[0] = 0;
  rs[0] = 0;
  for (int b = 0; b < nb; ++b) {
    n[b] = bn[b];
    del[b] = bdel ? bdel[b] : nullptr;
    ts[b + 1] = ts[b] + (bn[b] + kTile - 1) / kTile;
    rs[b + 1] = rs[b] + bn[b];
  }
  d.ntiles = ts[nb];
  d.rows = rs[nb];
  if (progs) {
    memcpy(st + oProg, progs, sizeof(TProgs));
    memcpy(st + oKinds, lay->kind, WS_MAX_AGGS);
    memcpy(st + oWoff, lay->woff, 4 * WS_MAX_AGGS);
    memcpy(st + oFwoff, lay->fwoff, 4 * WS_MAX_AGGS);
    memcpy(st + oNull, plan->aggNull, WS_MAX_AGGS);
    memcpy(st + oKeyInt, plan->keyInt, WS_MAX_KEYS);
  }
  d.buf = DBuf<uint8_t>((int64_t)off);
  h2dAsync(d.buf.p, st, off);
  stageCopied();
  uint8_t* p = d.buf.p;
  d.cols = (const ws_col_view*)(p + oCols);
  d.n = (const int64_t*)(p + oN);
  d.del = (const uint32_t* const*)(p + oDel);
  d.tileStart = (const int64_t*)(p + oTile);
  d.rowStart = (const int64_t*)(p + oRow);
  if (progs) {
    d.progs = (const TProgs*)(p + oProg);
    d.kinds = p + oKinds;
    d.woff = (const int*)(p + oWoff);
    d.fwoff = (const int*)(p + oFwoff);
    d.aggNull = p + oNull;
    d.keyInt = p + oKeyInt;
  }
  return d;
}

static void fillLaunch(Launch& L, const BatchDesc& d, int nb, int ncols, const ws_expr_env& env, const ws_agg_plan* plan,
                       const SlotLayout* lay) {
  memset(&L, 0, sizeof L);
  L.cols = d.cols;
  L.n = (const i64*)d.n;
  L.del = d.del;
  L.tileStart = (const i64*)d.tileStart;
  L.rowStart = (const i64*)d.rowStart;
  L.nb = nb;
  L.ncols = ncols;
  L.ntiles = d.ntiles;
  L.env = envK(env);
  L.progs = d.progs;
  L.kinds = d.kinds;
  L.woff = d.woff;
  L.fwoff = d.fwoff;
  L.aggNull = d.aggNull;
  L.keyInt = d.keyInt;
  if (plan) {
    L.nkeys = plan->nkeys;
    L.naggs = plan->naggs;
  }
  if (lay) {
    L.rowWords = lay->rw;
    L.fastWords = lay->frw;
  }
}

// A compiled plan can only run batches whose columns it was generated for: one generated for raw
// columns cannot decode an encoded segment (the engine's hint, env.cols[c].enc, says which may be).
static bool planCovers(const ws_expr_env& env, int nb, int ncols, const ws_col_view* bcols) {
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < ncols; ++c)
      if (bcols[(int64_t)b * ncols + c].enc && !env.cols[c].enc) return false;
  return true;
}

}  // namespace ws

using namespace ws;

// ================================================================ aggregation
struct ws_aggregator {
  ws_agg_plan plan{};
  ws_dense_spec dense{};
  bool isDense = false;
  SlotLayout lay;
  int64_t cap = 1;  // hash rows (power of two) / dense groups / 1
  int ncols = 0;
  std::vector<int64_t> bn;
  std::vector<const uint32_t*> bdel;
  std::vector<ws_col_view> bcols;
  int64_t rowsDone = 0;
  int batchesDone = 0, windows = 0;
  DBuf<u64> rows;
  DBuf<double> tkeys;
  DBuf<uint8_t> ctl;  // [count u64][err int x3][pad][ticket u32]
  bool fetched = false;
  std::vector<int64_t> hi;
  int64_t lastGroups = -1;
  // groups compacted on the device by the last fetch (reused by the copy after a size query, until
  // the next run): keys and engine-format doubles row-major, exact words [g][na][2]
  int64_t cachedGroups = -1;
  DBuf<double> cachedKeys, cachedAccs;
  DBuf<int64_t> cachedExact;
  std::vector<int64_t> cachedHi;
  // groups before each chunk of kOccChunk result rows (ws_agg_fetch_async), until the next run
  DBuf<int64_t> fetchOffs;
  bool fetchOffsValid = false;

  u64* count() { return (u64*)ctl.p; }
  int* err() { return (int*)(ctl.p + 8); }
  unsigned* ticket() { return (unsigned*)(ctl.p + 24); }
  int64_t nrows() const { return isDense ? dense.G : plan.nkeys ? cap + 1 : 1; }
};

namespace ws {

static RowTemplate rowTemplate(const SlotLayout& lay) {
  RowTemplate t{};
  for (int a = 0; a < lay.na; ++a) {
    const int o = lay.woff[a];
    switch (lay.kind[a]) {
      case SK_IMIN: t.w[o] = (u64)0x7fffffffffffffffll; break;
      case SK_IMAX: t.w[o] = (u64)0x8000000000000000ll; break;
      case SK_DMIN: {
        double inf = __builtin_inf();
        long long b;
        memcpy(&b, &inf, 8);
        t.w[o] = (u64)(b >= 0 ? b : (b ^ 0x7fffffffffffffffll));
        break;
      }
      case SK_DMAX: {
        double inf = -__builtin_inf();
        long long b;
        memcpy(&b, &inf, 8);
        t.w[o] = (u64)(b >= 0 ? b : (b ^ 0x7fffffffffffffffll));
        break;
      }
      default: break;
    }
  }
  return t;
}

// Result rows to their identities (hash rows empty) and the control words (count, flags, ticket) to 0.
static void aggResetRows(ws_aggregator& A) {
  const int64_t nr = A.nrows();
  const int64_t emptyRows = A.plan.nkeys && !A.isDense ? A.cap : 0;
  WS_LAUNCH(kFillRows, gridFor(nr), 256, 0, A.rows.p, nr, A.lay.rw, rowTemplate(A.lay), emptyRows);
  WS_CK(cudaMemsetAsync(A.ctl.p, 0, 32, stream()));
}

static void aggInitRows(ws_aggregator& A) {
  const int64_t nr = A.nrows();
  A.rows = DBuf<u64>(nr * A.lay.rw);
  if (A.plan.nkeys && !A.isDense) {
    A.tkeys = DBuf<double>((A.cap + 1) * std::max(A.plan.nkeys, 1));
  }
  A.ctl = DBuf<uint8_t>(32);
  aggResetRows(A);
}

static TuneChoice tuneScan(ws_aggregator& A, const std::string& key, const std::vector<TuneChoice>& cands,
                           const std::function<void(const TuneChoice&)>& launch);

// Default shared-memory budget of the hash scan's per-CTA table (KB; WARPSTORE_B200_HASH_SMEM_KB).
// 48 KB (1024 slots of a 32-byte row, 3 CTAs per SM with the spill buffer) measured 28 % faster than
// 64 KB on 100M Zipf-keyed rows (4.89 vs 6.79 ms) and the same on 16 groups, 6 groups and the
// serving workload's multi-key queries.
static int hashTableKB() {
  static const int kb = [] {
    const char* e = getenv("WARPSTORE_B200_HASH_SMEM_KB");
    const int v = e ? atoi(e) : 0;
    return v >= 4 && v <= 160 ? v : 48;
  }();
  return kb;
}

static size_t hashSmemSlots(const ws_aggregator& A, size_t budget) {
  const size_t per = (size_t)A.lay.rw * 8 + (A.plan.nkeys > 1 ? (size_t)A.plan.nkeys * 8 : 0);
  size_t s = 4096;
  while (s > 64 && s * per > budget) s >>= 1;
  return s * per > budget ? 0 : s;
}

// A scan prepared for launching elsewhere (a captured graph): kernel, shape, launch descriptor and the
// device buffers the descriptor points to.
struct PreparedScan {
  bool direct = false;    // in: direct loads only (a multi-query launch has no staged form)
  bool ready = false;     // false: the batches hold no tiles (nothing to launch)
  bool compiled = false;  // the plan's generated kernels (not the interpreter)
  CUfunction f = nullptr;
  unsigned grid = 0;
  size_t smem = 0;
  int threads = kThreads;
  Launch L{};
  BatchDesc desc;
  DBuf<u64> part;
};

// The aggregation scan over the collected batches; with `prep`, everything up to the launch (descriptor
// upload, kernel and shape choice, tuning) is done and the launch is handed to the caller instead.
static void aggRun(ws_aggregator& A, const ws_expr_env& env, const ws_jit_program* jit, PreparedScan* prep = nullptr) {
  const int nb = (int)A.bn.size();
  if (nb == 0) return;
  A.fetched = false;
  A.lastGroups = -1;
  A.cachedGroups = -1;
  A.fetchOffsValid = false;
  const bool useJit = jit && jit->state.load() == 1 && planCovers(env, nb, A.ncols, A.bcols.data());
  if (!useJit && (A.plan.naggs > WS_INTERP_AGGS || A.plan.nkeys > WS_INTERP_KEYS))
    throw Error("this aggregation needs a compiled plan (more than 16 aggregates or 4 GROUP BY keys); codegen failed or is off", WS_ERR_PLAN);
  std::unique_ptr<TProgs> progs;
  if (!useJit) {
    progs.reset(new TProgs);
    buildTProgs(env, A.ncols, A.plan, A.plan.hasWhere, *progs);
  }
  BatchDesc d = uploadBatches(nb, A.ncols, A.bn.data(), A.bdel.data(), A.bcols.data(), progs.get(), &A.lay, &A.plan);
  if (d.ntiles == 0) return;
  Launch L;
  fillLaunch(L, d, nb, A.ncols, env, &A.plan, &A.lay);
  L.rows = A.rows.p;
  L.err = A.err();
  L.ticket = A.ticket();
  const KernelSet& ks = useJit ? jit->kernels : interpKernels();
  // Staged scans: a ring of 2..4 tile stages in shared memory (compiled plans only).
  const int stageBytes = useJit ? jit->stageBytes : 0;
  static const int maxStages = [] {  // WARPSTORE_B200_STAGES: shared-memory tile stages (0: direct loads,
                                      // measured faster for the dense scan, which then fits 2 CTAs per SM)
    const char* e = getenv("WARPSTORE_B200_STAGES");
    return e ? std::max(0, std::min(8, atoi(e))) : 0;
  }();
  const int S = stageBytes > 0 ? (int)std::min<int64_t>(maxStages, (200 * 1024) / stageBytes) : 0;
  // The scan's launch shape as a function of a tuning choice: kernel, shared memory, block size and
  // the launch fields the shape changes.  Per-CTA partial rows (`part`: no-key and private-row scans)
  // are sized by the grid.
  struct Shape {
    CUfunction f = nullptr;
    size_t smem = 0;
    int threads = kThreads;
  };
  std::function<Shape(const TuneChoice&)> shapeOf;
  const char* name = "";
  int64_t partRows = 0;  // rows of `part` per CTA (0: none)
  std::vector<TuneChoice> cands(1);  // candidates for the autotuner; [0] = the default shape
  auto ctas = [](int c) {
    TuneChoice t;
    t.ctasPerSm = c;
    return t;
  };
  auto staged = [](int st) {
    TuneChoice t;
    t.stages = st;
    return t;
  };
  Launch* lp = &L;
  if (A.plan.nkeys == 0) {
    CUfunction f = ks.fn[K_NOKEYS];
    if (!f) throw Error("compiled plan has no aggregation kernel", WS_ERR_INTERNAL);
    shapeOf = [=](const TuneChoice& c) {
      // stage count: the choice's, else the default; within 200 KB of tile stages
      int st = c.stages >= 0 ? c.stages : S;
      if (stageBytes > 0) st = (int)std::min<int64_t>(st, (200 * 1024) / stageBytes);
      if (st < 2 || stageBytes <= 0) st = 0;
      lp->stages = st;
      return Shape{f, (size_t)st * stageBytes, st ? kStagedThreads : kThreads};
    };
    name = "nokeys";
    partRows = 1;
    cands.push_back(ctas(2));
    cands.push_back(ctas(1));
    if (stageBytes > 0)
      for (int st : {0, 2, 3})
        if (st != (S >= 2 ? S : 0)) cands.push_back(staged(st));
  } else if (A.isDense) {
    for (int k = 0; k < A.plan.nkeys; ++k) {
      L.kmin[k] = A.dense.kmin[k];
      L.range[k] = A.dense.range[k];
      L.stride[k] = A.dense.stride[k];
    }
    L.G = A.dense.G;
    const int64_t G = A.dense.G;
    // few groups: private register rows per thread in shared memory (+ staged tiles when they fit)
    // private rows [G][frw][kThreads] + int128 spill counters [G][NA][2] (NA: the evaluator's slot bound)
    const int naEv = ks.interp ? WS_INTERP_AGGS : A.plan.naggs;
    const size_t privBytes = (size_t)G * A.lay.frw * kThreads * 8 + (size_t)G * naEv * 16;
    const size_t sharedSmem = (size_t)G * A.lay.rw * 8;
    if (G * A.lay.frw <= 48 && ks.fn[K_DENSE_PRIV]) {
      // tile stages fit beside the private rows within 220 KB; the staged body is its own entry
      const int64_t room = std::max<int64_t>(0, (int64_t)(220 * 1024) - (int64_t)privBytes);
      const int fitStages = stageBytes > 0 ? (int)std::min<int64_t>(8, room / stageBytes) : 0;
      CUfunction direct = ks.fn[K_DENSE_PRIV], stagedFn = ks.fn[K_DENSE_PRIV_STAGED];
      shapeOf = [=](const TuneChoice& c) {
        int st = std::min(c.stages >= 0 ? c.stages : maxStages, fitStages);
        if (st < 2 || !stagedFn) st = 0;
        lp->stages = st;
        return Shape{st ? stagedFn : direct, (size_t)st * stageBytes + privBytes, st ? kStagedThreads : kThreads};
      };
      name = "dense_priv";
      partRows = G;
      cands.push_back(ctas(1));
      if (stagedFn && fitStages >= 2)
        for (int st : {0, 2, 3})
          if (st <= fitStages && st != (std::min(maxStages, fitStages) >= 2 ? std::min(maxStages, fitStages) : 0))
            cands.push_back(staged(st));
    } else if (sharedSmem <= 96 * 1024 && ks.fn[K_DENSE_SHARED]) {
      CUfunction f = ks.fn[K_DENSE_SHARED];
      shapeOf = [=](const TuneChoice&) { return Shape{f, sharedSmem, kThreads}; };
      name = "dense_shared";
      cands.push_back(ctas(2));
      cands.push_back(ctas(1));
    } else {
      CUfunction f = ks.fn[K_DENSE_GLOBAL];
      if (!f) throw Error("compiled plan has no dense kernel", WS_ERR_INTERNAL);
      shapeOf = [=](const TuneChoice&) { return Shape{f, 0, kThreads}; };
      name = "dense_global";
      cands.push_back(ctas(4));
      cands.push_back(ctas(2));
    }
  } else {
    CUfunction f = ks.fn[K_HASH];
    if (!f) throw Error("compiled plan has no hash aggregation kernel", WS_ERR_INTERNAL);
    L.table = A.rows.p;
    L.tkeys = A.tkeys.p;
    L.mask = (u64)(A.cap - 1);
    L.count = A.count();
    L.probeLimit = (int)std::min<int64_t>(A.cap, 1 << 16);
    const size_t per = (size_t)A.lay.rw * 8 + (A.plan.nkeys > 1 ? (size_t)A.plan.nkeys * 8 : 0);
    // spill buffer: up to a tile's rows, within 40 KB
    L.spillRows = (int)std::min<size_t>(kTile, (40 * 1024) / per);
    ws_aggregator* ap = &A;
    shapeOf = [=](const TuneChoice& c) {
      // per-CTA table: up to 4096 slots within the budget (default 64 KB)
      const size_t slots = hashSmemSlots(*ap, (size_t)(c.smemKB > 0 ? c.smemKB : hashTableKB()) * 1024);
      lp->smemSlots = (int)slots;
      return Shape{f, (slots + (size_t)lp->spillRows) * per, kThreads};
    };
    name = "hash";
    for (int kb : {16, 32, 96}) {
      TuneChoice t;
      t.smemKB = kb;
      cands.push_back(t);
    }
    cands.push_back(ctas(2));
  }
  DBuf<u64> part;
  int64_t partCap = 0;
  auto launchOnce = [&](const TuneChoice& c) {
    const Shape sh = shapeOf(c);
    unsigned grid = persistentGrid(sh.f, sh.smem, d.ntiles, sh.threads);
    if (c.ctasPerSm > 0) grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)c.ctasPerSm * smCount()));
    if (partRows) {
      if ((int64_t)grid * partRows > partCap) {
        partCap = (int64_t)grid * partRows;
        part = DBuf<u64>(partCap * A.lay.rw);
      }
      L.part = part.p;
      WS_CK(cudaMemsetAsync(A.ticket(), 0, 4, stream()));
    }
    launchScan(sh.f, grid, sh.smem, L, sh.threads);
  };
  const std::string key = tuneKey(name, useJit ? jit : nullptr, A.plan, d.ntiles);
  TuneChoice choice;
  if (prep && prep->direct) {  // tuned without staged candidates: a multi-query launch loads directly
    std::vector<TuneChoice> directOnly;
    for (const TuneChoice& c : cands)
      if (c.stages <= 0) directOnly.push_back(c);
    for (TuneChoice& c : directOnly) c.stages = 0;
    cands.swap(directOnly);
  }
  if (!tuneLookup(key, choice) && tuneMode() == WS_TUNE_ON && A.windows == 0 && A.rowsDone == 0)
    choice = tuneScan(A, key, cands, launchOnce);
  if (prep && prep->direct) choice.stages = 0;
  if (prep) {
    const Shape sh = shapeOf(choice);
    unsigned grid = persistentGrid(sh.f, sh.smem, d.ntiles, sh.threads);
    if (choice.ctasPerSm > 0)
      grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)choice.ctasPerSm * smCount()));
    if (partRows) {
      part = DBuf<u64>((int64_t)grid * partRows * A.lay.rw);
      L.part = part.p;
    }
    prep->compiled = useJit;
    prep->f = sh.f;
    prep->grid = grid;
    prep->smem = sh.smem;
    prep->threads = sh.threads;
    prep->L = L;
    prep->L.sumShift = sumShiftFor(L.ntiles, grid);
    prep->L.waitLog2 = stagedWaitLog2();
    prep->desc = std::move(d);
    prep->part = std::move(part);
    prep->ready = true;
    return;
  }
  launchOnce(choice);
}

// Times each candidate launch shape of a scan on the aggregation's own batches (best of two runs,
// CUDA events on the calling stream, the result rows reset before each run) and records the fastest;
// the rows are reset again for the caller's final run.  A run that raised a flag (overflow, key out of
// range) records nothing: the final run raises it again and the caller decides.
static TuneChoice tuneScan(ws_aggregator& A, const std::string& key, const std::vector<TuneChoice>& cands,
                           const std::function<void(const TuneChoice&)>& launch) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WS_CK(cudaEventCreate(&e0));
  WS_CK(cudaEventCreate(&e1));
  TuneChoice best;
  double bestMs = 1e300;
  bool flagged = false;
  try {
    for (const TuneChoice& c : cands) {
      double ms = 1e300;
      for (int rep = 0; rep < 2; ++rep) {
        aggResetRows(A);
        WS_CK(cudaEventRecord(e0, stream()));
        launch(c);
        WS_CK(cudaEventRecord(e1, stream()));
        WS_CK(cudaEventSynchronize(e1));
        float t = 0;
        WS_CK(cudaEventElapsedTime(&t, e0, e1));
        ms = std::min(ms, (double)t);
      }
      int e[3] = {0, 0, 0};
      d2hSync(e, A.err(), 12);
      flagged |= e[0] || e[1] || e[2];
      if (ms < bestMs) bestMs = ms, best = c;
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  aggResetRows(A);
  if (flagged) return TuneChoice{};
  tuneStore(key, best, bestMs * 1000);
  best.found = true;
  return best;
}

// Occupied row indices of the result rows (ascending), on the device; returns the count.
static int64_t aggCompactIdx(ws_aggregator& A, DBuf<int64_t>& idx) {
  const int64_t nr = A.nrows();
  OccSpec s{A.lay.rw, A.isDense ? 1 : 2, A.lay.woff[0], A.cap};
  const int64_t nchunks = (nr + kOccChunk - 1) / kOccChunk;
  DBuf<int64_t> counts(nchunks + 1);
  WS_LAUNCH(kOccCount, (unsigned)nchunks, 256, 0, A.rows.p, nr, s, counts.p);
  WS_LAUNCH(kScanExclusive, 1, 1024, 0, counts.p, nchunks);
  int64_t g = 0;
  d2hSync(&g, counts.p + nchunks, 8);
  idx = DBuf<int64_t>(std::max<int64_t>(g, 1));
  if (g) WS_LAUNCH(kOccWrite, (unsigned)nchunks, 256, 0, A.rows.p, nr, s, counts.p, idx.p);
  return g;
}

static EmitSpec emitSpec(const ws_aggregator& A) {
  EmitSpec s{};
  s.nk = A.plan.nkeys;
  s.na = A.plan.naggs;
  s.rw = A.lay.rw;
  s.mode = A.plan.nkeys == 0 ? 0 : A.isDense ? 1 : 2;
  for (int a = 0; a < s.na; ++a) {
    s.kind[a] = A.lay.kind[a];
    s.woff[a] = (int16_t)A.lay.woff[a];
    s.partner[a] = (int16_t)A.lay.partner[a];
  }
  for (int k = 0; k < s.nk; ++k) {
    s.keyInt[k] = A.plan.keyInt[k];
    s.kmin[k] = A.dense.kmin[k];
    s.range[k] = A.isDense ? A.dense.range[k] : 1;
    s.stride[k] = A.isDense ? A.dense.stride[k] : 1;
  }
  s.tkeys = A.tkeys.p;
  s.cap = A.cap;
  return s;
}

static DblSpec dblSpec(const ws_aggregator& A) {
  DblSpec s{};
  s.na = A.plan.naggs;
  s.nokeys = A.plan.nkeys == 0;
  for (int a = 0; a < s.na; ++a) {
    s.kind[a] = A.lay.kind[a];
    s.aggBits[a] = A.plan.aggBits[a];
    s.aggPart[a] = A.plan.aggPart[a];
  }
  return s;
}

static void checkFlags(ws_aggregator& A, bool* overflow) {
  int e[3] = {0, 0, 0};
  d2hSync(e, A.err(), 12);
  if (e[0]) throw Error("dense GROUP BY key outside its declared range", WS_ERR_RANGE);
  if (e[2]) throw Error("a staged tile copy did not complete in time", WS_ERR_INTERNAL);
  if (overflow) *overflow = e[1] != 0;
}

// One multi-query scan over prepared queries (ws_agg_run_many, ws_exec_group_*): the kernel of the
// queries' common scan kind, its shared memory and block, the queries that have tiles, their CTA
// starts (the launch's resident CTAs shared out by tiles: each query at least one CTA, at most its own
// persistent grid, which its partial rows were sized for) and their launch descriptors.
struct MultiPlan {
  CUfunction f = nullptr;
  size_t smem = 0;
  int threads = 0;
  std::vector<int> live;    // indices of the queries with tiles
  std::vector<int> start;   // CTA starts, live.size() + 1
  std::vector<Launch> L;    // per live query, ctaBase / ctaGrid left for the kernel
};

static MultiPlan planMulti(const std::vector<const PreparedScan*>& preps, const ws_jit_program* jit, const char* who) {
  MultiPlan mp;
  const KernelSet* ks = nullptr;
  int multi = -1;
  int64_t tiles = 0;
  for (size_t i = 0; i < preps.size(); ++i) {
    const PreparedScan& p = *preps[i];
    if (!p.ready) continue;  // no tiles: nothing to scan
    if (p.compiled && !jit) throw Error(std::string(who) + ": compiled queries need their plan", WS_ERR_ARG);
    const KernelSet& k = p.compiled ? jit->kernels : interpKernels();
    const int m = p.f == k.fn[K_NOKEYS] ? K_MULTI_NOKEYS : p.f == k.fn[K_DENSE_PRIV] ? K_MULTI_DENSE_PRIV
                : p.f == k.fn[K_HASH] ? K_MULTI_HASH : -1;
    if (m < 0 || !k.fn[m] || p.L.stages)
      throw Error(std::string(who) + ": a query's scan has no multi-query form (dense shared / global rows, staged tiles)",
                  WS_ERR_ARG);
    if (multi >= 0 && (m != multi || &k != ks))
      throw Error(std::string(who) + ": the queries need one scan kind and one plan (or all interpreted)", WS_ERR_ARG);
    ks = &k, multi = m;
    mp.smem = std::max(mp.smem, p.smem);
    mp.threads = p.threads;
    tiles += p.L.ntiles;
    mp.live.push_back((int)i);
  }
  if (mp.live.empty()) return mp;
  mp.f = ks->fn[multi];
  const unsigned total = persistentGrid(mp.f, mp.smem, std::max<int64_t>(tiles, (int64_t)mp.live.size()), mp.threads);
  mp.start.assign(mp.live.size() + 1, 0);
  for (size_t j = 0; j < mp.live.size(); ++j) {
    const PreparedScan& p = *preps[(size_t)mp.live[j]];
    int64_t share = (int64_t)((double)total * (double)p.L.ntiles / (double)tiles);
    share = std::max<int64_t>(1, std::min<int64_t>(share, std::min<int64_t>(p.grid, p.L.ntiles)));
    mp.start[j + 1] = mp.start[j] + (int)share;
    Launch L = p.L;
    L.sumShift = sumShiftFor(L.ntiles, (unsigned)share);
    L.waitLog2 = stagedWaitLog2();
    L.ctaBase = L.ctaGrid = 0;  // set per CTA by the kernel
    mp.L.push_back(L);
  }
  return mp;
}

}  // namespace ws

extern "C" {

int ws_agg_create(const ws_agg_plan* plan, int64_t capacity, const ws_dense_spec* dense, ws_aggregator** out) {
  return guardedCall([&] {
    *out = nullptr;
    std::unique_ptr<ws_aggregator> A(new ws_aggregator);
    A->plan = *plan;
    A->lay = layoutOf(*plan);
    if (dense && dense->G > 0 && plan->nkeys) {
      A->dense = *dense;
      A->isDense = true;
      A->cap = dense->G;
    } else if (plan->nkeys) {
      int64_t c = 1;
      while (c < capacity) c <<= 1;
      A->cap = std::max<int64_t>(c, 2);
    } else {
      A->cap = 1;
    }
    aggInitRows(*A);
    *out = A.release();
  });
}

void ws_agg_destroy(ws_aggregator* agg) { delete agg; }

int ws_agg_add_batch(ws_aggregator* A, const ws_expr_env* env, int ncols, int64_t n, const uint32_t* del) {
  return guardedCall([&] {
    if (n <= 0) return;
    if (ncols < 0 || ncols > WS_MAX_COLS) throw Error("bad column count", WS_ERR_ARG);
    if (!A->bn.empty() && ncols != A->ncols) throw Error("batches must have the same column count", WS_ERR_ARG);
    A->ncols = ncols;
    A->bn.push_back(n);
    A->bdel.push_back(del);
    for (int i = 0; i < ncols; ++i) A->bcols.push_back(env->cols[i]);
  });
}

int ws_agg_add_batches(ws_aggregator* A, int ncols, int nb, const int64_t* bn, const uint32_t* const* bdel,
                       const ws_col_view* bcols) {
  return guardedCall([&] {
    if (ncols < 0 || ncols > WS_MAX_COLS || nb < 0) throw Error("bad column or batch count", WS_ERR_ARG);
    for (int b = 0; b < nb; ++b) {
      if (bn[b] <= 0) continue;
      if (!A->bn.empty() && ncols != A->ncols) throw Error("batches must have the same column count", WS_ERR_ARG);
      A->ncols = ncols;
      A->bn.push_back(bn[b]);
      A->bdel.push_back(bdel ? bdel[b] : nullptr);
      A->bcols.insert(A->bcols.end(), bcols + (int64_t)b * ncols, bcols + (int64_t)(b + 1) * ncols);
    }
  });
}

int ws_agg_run(ws_aggregator* A, const ws_expr_env* env, const ws_jit_program* jit) {
  return guardedCall([&] { aggRun(*A, *env, jit); });
}

int ws_agg_run_many(ws_aggregator* const* aggs, const ws_expr_env* const* envs, const ws_jit_program* jit, int n) {
  return guardedCall([&] {
    if (n < 1 || n > 1024 || !aggs || !envs) throw Error("ws_agg_run_many: 1..1024 aggregators", WS_ERR_ARG);
    // each query prepared as for its own launch (descriptor uploaded, kernel and shape chosen)
    std::vector<PreparedScan> preps((size_t)n);
    for (int i = 0; i < n; ++i) {
      preps[(size_t)i].direct = true;
      aggRun(*aggs[i], *envs[i], jit, &preps[(size_t)i]);
    }
    std::vector<const PreparedScan*> pp;
    for (const PreparedScan& p : preps) pp.push_back(&p);
    const MultiPlan mp = planMulti(pp, jit, "ws_agg_run_many");
    if (mp.live.empty()) return;
    const size_t nl = mp.live.size();
    const size_t launchBytes = nl * sizeof(Launch), startBytes = (nl + 1) * sizeof(int);
    uint8_t* st = pinnedStage(launchBytes + startBytes);
    memcpy(st, mp.L.data(), launchBytes);
    memcpy(st + launchBytes, mp.start.data(), startBytes);
    for (const Launch& L : mp.L)
      if (L.ticket) WS_CK(cudaMemsetAsync(L.ticket, 0, 4, stream()));
    DBuf<uint8_t> dl((int64_t)(launchBytes + startBytes));
    h2dAsync(dl.p, st, launchBytes + startBytes);
    stageCopied();
    MultiLaunch M{(const Launch*)dl.p, (const int*)(dl.p + launchBytes), (int)nl};
    allowDynamicSmem(mp.f, mp.smem);
    void* args[] = {(void*)&M};
    WS_CKD(drv().launchKernel(mp.f, (unsigned)mp.start[nl], 1, 1, (unsigned)mp.threads, 1, 1, (unsigned)mp.smem,
                              (CUstream)stream(), args, nullptr));
    countLaunch();
  });
}

int ws_agg_run_window(ws_aggregator* A, const ws_expr_env* env, const ws_jit_program* jit) {
  return guardedCall([&] {
    if (A->bn.empty()) return;
    aggRun(*A, *env, jit);
    ++A->windows;
    for (int64_t n : A->bn) A->rowsDone += n;
    A->batchesDone += (int)A->bn.size();
    A->bn.clear();
    A->bdel.clear();
    A->bcols.clear();
  });
}

int ws_agg_batches(const ws_aggregator* A) { return A->batchesDone + (int)A->bn.size(); }
int ws_agg_windows(const ws_aggregator* A) { return A->windows; }
int64_t ws_agg_rows_in(const ws_aggregator* A) {
  int64_t r = A->rowsDone;
  for (int64_t n : A->bn) r += n;
  return r;
}
int ws_agg_is_dense(const ws_aggregator* A) { return A->isDense ? 1 : 0; }
int64_t ws_agg_capacity(const ws_aggregator* A) { return A->cap; }

int ws_agg_overflowed(ws_aggregator* A, int* out) {
  return guardedCall([&] {
    bool o = false;
    checkFlags(*A, &o);
    *out = A->plan.nkeys && !A->isDense && o ? 1 : 0;
  });
}

int ws_agg_group_count(ws_aggregator* A, int64_t* out) {
  return guardedCall([&] {
    if (!A->plan.nkeys) {
      *out = 1;
      return;
    }
    if (A->isDense) {
      DBuf<int64_t> idx;
      *out = aggCompactIdx(*A, idx);
      return;
    }
    u64 c = 0;
    d2hSync(&c, A->count(), 8);
    *out = (int64_t)c;
  });
}

int ws_agg_fetch(ws_aggregator* A, int64_t max_groups, double* keys, double* accs, int64_t* exact, int64_t* ngroups) {
  return guardedCall([&] {
    const int nk = A->plan.nkeys, na = A->plan.naggs;
    if (A->cachedGroups < 0) {  // compact and convert on the device once; the copy after a size query reuses it
      checkFlags(*A, nullptr);
      DBuf<int64_t> idx;
      const int64_t g = nk ? aggCompactIdx(*A, idx) : 1;
      A->cachedKeys = DBuf<double>(std::max<int64_t>(g * nk, 1));
      A->cachedExact = DBuf<int64_t>(std::max<int64_t>(g * na * 2, 1));
      A->cachedAccs = DBuf<double>(std::max<int64_t>(g * na, 1));
      if (g) {
        WS_LAUNCH(kEmit, gridFor(g), 256, 0, A->rows.p, nk ? idx.p : nullptr, g, emitSpec(*A), A->cachedKeys.p,
                  A->cachedExact.p, 0);
        DBuf<int16_t> pk(WS_MAX_AGGS);
        int16_t* st = (int16_t*)pinnedStage(2 * WS_MAX_AGGS);
        for (int a = 0; a < WS_MAX_AGGS; ++a) st[a] = a < na ? A->lay.kind[A->lay.partner[a]] : 0;
        h2dAsync(pk.p, st, 2 * WS_MAX_AGGS);
        stageCopied();
        WS_LAUNCH(kExactToDouble, gridFor(g), 256, 0, A->cachedExact.p, g, dblSpec(*A), pk.p, A->cachedAccs.p, 0);
      }
      A->cachedHi.assign(na, 0);
      if (!nk) {  // high words of exact no-key integer sums (sumHigh)
        std::vector<int64_t> ex(2 * na);
        d2hSync(ex.data(), A->cachedExact.p, 16 * na);
        for (int a = 0; a < na; ++a) {
          const uint8_t k = A->lay.kind[a] == SK_NONE ? A->lay.kind[A->lay.partner[a]] : A->lay.kind[a];
          A->cachedHi[a] = k == SK_ISUM ? ex[2 * a + 1] : 0;
        }
      } else {
        sync();
      }
      A->cachedGroups = g;
    }
    const int64_t g = A->cachedGroups;
    *ngroups = g;
    if (g > max_groups) throw Error("output buffer too small for " + std::to_string(g) + " groups", WS_ERR_SIZE);
    if (g) {
      if (nk && keys) d2hLarge(keys, A->cachedKeys.p, sizeof(double) * g * nk);
      if (accs) d2hLarge(accs, A->cachedAccs.p, sizeof(double) * g * na);
      if (exact) d2hLarge(exact, A->cachedExact.p, sizeof(int64_t) * g * na * 2);
    }
    A->hi = A->cachedHi;
    A->fetched = true;
  });
}

int ws_agg_fetch_async(ws_aggregator* A, int64_t first_group, int64_t max_groups, double* keys, int64_t* exact,
                       ws_fetch_status* status) {
  return guardedCall([&] {
    const int nk = A->plan.nkeys, na = A->plan.naggs;
    auto mapped = [](void* h, const char* what) -> void* {
      if (!h) throw Error(std::string("fetch_async: ") + what + " is null", WS_ERR_ARG);
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, h) != cudaSuccess || at.type != cudaMemoryTypeHost || !at.devicePointer) {
        cudaGetLastError();
        throw Error(std::string("fetch_async: ") + what + " is not pinned host memory", WS_ERR_ARG);
      }
      return at.devicePointer;
    };
    auto* st = (ws_fetch_status*)mapped(status, "status");
    double* dk = nk ? (double*)mapped(keys, "keys") : nullptr;
    auto* dx = (long long*)mapped(exact, "exact");
    if (first_group < 0 || max_groups < 0) throw Error("fetch_async: negative group range", WS_ERR_ARG);
    const int64_t nr = A->nrows();
    OccSpec o{A->lay.rw, nk == 0 ? 0 : A->isDense ? 1 : 2, A->lay.woff[0], A->cap};
    const int64_t nchunks = (nr + kOccChunk - 1) / kOccChunk;
    if (!A->fetchOffsValid) {  // group offsets per chunk, kept for the later ranges of the same run
      A->fetchOffs = DBuf<int64_t>(nchunks + 1);
      WS_LAUNCH(kOccCount, (unsigned)nchunks, 256, 0, A->rows.p, nr, o, A->fetchOffs.p);
      WS_LAUNCH(kScanExclusive, 1, 1024, 0, A->fetchOffs.p, nchunks);
      A->fetchOffsValid = true;
    }
    const int64_t* counts = A->fetchOffs.p;
    WS_LAUNCH(kFetchStatus, 1, 1, 0, counts + nchunks, A->err(), o.mode == 2 ? 1 : 0, st);
    if (max_groups == 0) return;
    // sub-tile rows: staging of at most 32 KB, a multiple of 32 rows
    const int rowBytes = 8 * (nk + 2 * na);
    const int threads = std::max(32, std::min(256, (32768 / rowBytes) & ~31));
    WS_LAUNCH(kOccEmitHost, (unsigned)nchunks, threads, (size_t)threads * rowBytes, A->rows.p, nr, o, emitSpec(*A),
              counts, nchunks, A->err(), first_group, max_groups, dk, dx);
    A->cachedGroups = -1;
    A->fetched = true;
  });
}

}  // extern "C"

// A prepared query (ws_exec_*): the aggregation's result rows, its batch descriptor and one CUDA graph
// of the whole query — result rows reset, the scan, compaction, the groups and the status written into
// pinned host memory — captured once; each run updates the scan node's launch descriptor (the plan's
// constants) and launches the graph.
struct ws_executor {
  ws_aggregator* A = nullptr;
  ws::PreparedScan ps;
  uint64_t code = 0;  // digest of the expressions the graph was built for
  int64_t maxGroups = 0;
  double* keys = nullptr;
  int64_t* exact = nullptr;
  ws_fetch_status* st = nullptr;
  ws::DBuf<int64_t> offs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t scanNode = nullptr;
  int kernels = 0;  // kernel nodes per run
  ~ws_executor() {
    cudaStreamSynchronize(ws::stream());  // a run queued on this thread's stream may still be in flight
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (keys) cudaFreeHost(keys);
    if (exact) cudaFreeHost(exact);
    if (st) cudaFreeHost(st);
    if (A) ws_agg_destroy(A);
  }
};

namespace {
// Queues on this thread's stream the part of a prepared query after its scan: compaction of the
// result rows, the status word and the groups written into the executor's pinned memory.
void queueExecTail(ws_executor& X) {
  ws_aggregator& A = *X.A;
  const int nk = A.plan.nkeys, na = A.plan.naggs;
  double* dk = nullptr;
  long long* dx = nullptr;
  ws_fetch_status* dst = nullptr;
  WS_CK(cudaHostGetDevicePointer((void**)&dk, X.keys, 0));
  WS_CK(cudaHostGetDevicePointer((void**)&dx, X.exact, 0));
  WS_CK(cudaHostGetDevicePointer((void**)&dst, X.st, 0));
  const int64_t nr = A.nrows();
  const OccSpec o{A.lay.rw, nk == 0 ? 0 : A.isDense ? 1 : 2, A.lay.woff[0], A.cap};
  const int64_t nchunks = (nr + kOccChunk - 1) / kOccChunk;
  const int rowBytes = 8 * (nk + 2 * na);
  const int threads = std::max(32, std::min(256, (32768 / rowBytes) & ~31));
  WS_LAUNCH(kOccCount, (unsigned)nchunks, 256, 0, A.rows.p, nr, o, X.offs.p);
  WS_LAUNCH(kScanExclusive, 1, 1024, 0, X.offs.p, nchunks);
  WS_LAUNCH(kFetchStatus, 1, 1, 0, X.offs.p + nchunks, A.err(), o.mode == 2 ? 1 : 0, dst);
  WS_LAUNCH(kOccEmitHost, (unsigned)nchunks, threads, (size_t)threads * rowBytes, A.rows.p, nr, o, emitSpec(A), X.offs.p,
            nchunks, A.err(), (int64_t)0, X.maxGroups, dk, dx);
}

uint64_t codeDigest(const ws_expr_env& env) {
  uint64_t h = 0xcbf29ce484222325ull;
  const unsigned char* b = (const unsigned char*)env.code;
  for (size_t i = 0; i < sizeof env.code; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}
}  // namespace

extern "C" {

int ws_exec_create(const ws_agg_plan* plan, int64_t capacity, const ws_dense_spec* dense, const ws_expr_env* env,
                   int ncols, int nb, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                   const ws_jit_program* jit, int64_t max_groups, ws_executor** out) {
  return guardedCall([&] {
    *out = nullptr;
    if (max_groups < 1) throw Error("exec: max_groups must be positive", WS_ERR_ARG);
    if (!jit || jit->state.load() != 1) throw Error("exec: a prepared query needs a compiled plan", WS_ERR_PLAN);
    std::unique_ptr<ws_executor> X(new ws_executor);
    if (int rc = ws_agg_create(plan, capacity, dense, &X->A)) throw Error(ws_last_error(), rc);
    if (int rc = ws_agg_add_batches(X->A, ncols, nb, bn, bdel, bcols)) throw Error(ws_last_error(), rc);
    ws_aggregator& A = *X->A;
    aggRun(A, *env, jit, &X->ps);
    if (X->ps.ready && !X->ps.compiled)
      throw Error("exec: the compiled plan does not cover these batches (encodings)", WS_ERR_PLAN);
    X->code = codeDigest(*env);
    X->maxGroups = max_groups;
    const int nk = A.plan.nkeys, na = A.plan.naggs;
    auto pinned = [](size_t bytes, void** p) {
      if (cudaHostAlloc(p, std::max<size_t>(bytes, 8), cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        throw Error("exec: pinned result buffers", WS_ERR_OOM);
      }
    };
    pinned(sizeof(double) * max_groups * std::max(nk, 1), (void**)&X->keys);
    pinned(sizeof(int64_t) * max_groups * na * 2, (void**)&X->exact);
    pinned(sizeof(ws_fetch_status), (void**)&X->st);
    X->offs = DBuf<int64_t>((A.nrows() + kOccChunk - 1) / kOccChunk + 1);
    sync();  // the preparation's copies and allocations are done before the capture starts
    // capture on a private stream (nothing else of this thread's work joins the graph)
    cudaStream_t cs = nullptr;
    WS_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaStream_t prev = stream();
    auto restore = [&] { ws_set_stream(prev == cudaStreamPerThread ? nullptr : (void*)prev); };
    ws_set_stream(cs);
    bool capturing = false;
    try {
      WS_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      capturing = true;
      aggResetRows(A);
      X->kernels = 1;
      if (X->ps.ready) {
        const PreparedScan& p = X->ps;
        allowDynamicSmem(p.f, p.smem);
        void* args[] = {(void*)&X->ps.L};
        WS_CKD(drv().launchKernel(p.f, p.grid, 1, 1, (unsigned)p.threads, 1, 1, (unsigned)p.smem, (CUstream)cs, args,
                                  nullptr));
        countLaunch();
        cudaStreamCaptureStatus cst;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        WS_CK(cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &ndeps));
        if (ndeps != 1) throw Error("exec: could not find the scan in the captured graph", WS_ERR_INTERNAL);
        X->scanNode = deps[0];
        ++X->kernels;
      }
      queueExecTail(*X);
      X->kernels += 4;
      capturing = false;
      WS_CK(cudaStreamEndCapture(cs, &X->graph));
      WS_CK(cudaGraphInstantiate(&X->exec, X->graph, 0));
    } catch (...) {
      if (capturing) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
      }
      restore();
      cudaStreamDestroy(cs);
      throw;
    }
    countLaunch(-X->kernels);  // captured, not launched
    restore();
    WS_CK(cudaStreamDestroy(cs));
    *out = X.release();
  });
}

int ws_exec_run(ws_executor* X, const ws_expr_env* env) {
  return guardedCall([&] {
    if (codeDigest(*env) != X->code) throw Error("exec: the expressions differ from the prepared query's", WS_ERR_ARG);
    if (X->scanNode) {
      X->ps.L.env = envK(*env);
      void* args[] = {(void*)&X->ps.L};
      CUDA_KERNEL_NODE_PARAMS kp{};
      kp.func = X->ps.f;
      kp.gridDimX = X->ps.grid;
      kp.gridDimY = kp.gridDimZ = 1;
      kp.blockDimX = (unsigned)X->ps.threads;
      kp.blockDimY = kp.blockDimZ = 1;
      kp.sharedMemBytes = (unsigned)X->ps.smem;
      kp.kernelParams = args;
      WS_CKD(drv().graphExecKernelNodeSetParams((CUgraphExec)X->exec, (CUgraphNode)X->scanNode, &kp));
    }
    WS_CK(cudaGraphLaunch(X->exec, stream()));
    countLaunch(X->kernels);
  });
}

int ws_exec_results(ws_executor* X, const double** keys, const int64_t** exact, const ws_fetch_status** status) {
  if (keys) *keys = X->keys;
  if (exact) *exact = X->exact;
  if (status) *status = X->st;
  return WS_OK;
}

void ws_exec_destroy(ws_executor* X) { delete X; }

}  // extern "C"

// Prepared queries of one plan run together (ws_exec_group_*): one CUDA graph that resets every
// query's result rows, copies the queries' launch descriptors from pinned memory (each run writes the
// new constants there first), runs ONE multi-query scan over all of them and then each query's
// compaction and delivery into its own executor's pinned memory.
struct ws_exec_group {
  std::vector<ws_executor*> xs;
  ws::MultiPlan mp;
  uint8_t* stage = nullptr;  // pinned: [Launch per live query][CTA starts]
  size_t stageBytes = 0;
  ws::DBuf<uint8_t> dl;      // the device copy the scan reads
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;  // the last run's end: its copy of `stage` has been made
  int kernels = 0;
  ~ws_exec_group() {
    if (done) cudaEventSynchronize(done);
    cudaStreamSynchronize(ws::stream());
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (done) cudaEventDestroy(done);
    if (stage) cudaFreeHost(stage);
  }
};

extern "C" {

int ws_exec_group_create(ws_executor* const* xs, int n, const ws_jit_program* jit, ws_exec_group** out) {
  return guardedCall([&] {
    *out = nullptr;
    if (n < 1 || n > 1024 || !xs) throw Error("exec group: 1..1024 prepared queries", WS_ERR_ARG);
    std::unique_ptr<ws_exec_group> G(new ws_exec_group);
    std::vector<const PreparedScan*> pp;
    for (int i = 0; i < n; ++i) {
      if (!xs[i]) throw Error("exec group: a null prepared query", WS_ERR_ARG);
      for (int j = 0; j < i; ++j)
        if (xs[j] == xs[i]) throw Error("exec group: a prepared query given twice", WS_ERR_ARG);
      G->xs.push_back(xs[i]);
      pp.push_back(&xs[i]->ps);
    }
    G->mp = planMulti(pp, jit, "exec group");
    const MultiPlan& mp = G->mp;
    const size_t nl = mp.live.size();
    const size_t launchBytes = nl * sizeof(Launch), startBytes = (nl + 1) * sizeof(int);
    G->stageBytes = launchBytes + startBytes;
    if (cudaHostAlloc((void**)&G->stage, std::max<size_t>(G->stageBytes, 8), cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      G->stage = nullptr;
      throw Error("exec group: pinned descriptor buffer", WS_ERR_OOM);
    }
    if (nl) {
      memcpy(G->stage, mp.L.data(), launchBytes);
      memcpy(G->stage + launchBytes, mp.start.data(), startBytes);
      G->dl = DBuf<uint8_t>((int64_t)G->stageBytes);
    }
    WS_CK(cudaEventCreateWithFlags(&G->done, cudaEventDisableTiming));
    sync();  // allocations done before the capture starts
    cudaStream_t cs = nullptr;
    WS_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaStream_t prev = stream();
    auto restore = [&] { ws_set_stream(prev == cudaStreamPerThread ? nullptr : (void*)prev); };
    ws_set_stream(cs);
    const int64_t launches0 = ws_kernel_launches();
    bool capturing = false;
    try {
      WS_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      capturing = true;
      for (ws_executor* X : G->xs) aggResetRows(*X->A);
      if (nl) {
        WS_CK(cudaMemcpyAsync(G->dl.p, G->stage, G->stageBytes, cudaMemcpyHostToDevice, cs));
        for (const Launch& L : mp.L)
          if (L.ticket) WS_CK(cudaMemsetAsync(L.ticket, 0, 4, cs));
        MultiLaunch M{(const Launch*)G->dl.p, (const int*)(G->dl.p + launchBytes), (int)nl};
        allowDynamicSmem(mp.f, mp.smem);
        void* args[] = {(void*)&M};
        WS_CKD(drv().launchKernel(mp.f, (unsigned)mp.start[nl], 1, 1, (unsigned)mp.threads, 1, 1, (unsigned)mp.smem,
                                  (CUstream)cs, args, nullptr));
        countLaunch();
      }
      for (ws_executor* X : G->xs) queueExecTail(*X);
      capturing = false;
      WS_CK(cudaStreamEndCapture(cs, &G->graph));
      WS_CK(cudaGraphInstantiate(&G->exec, G->graph, 0));
    } catch (...) {
      if (capturing) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
      }
      restore();
      cudaStreamDestroy(cs);
      throw;
    }
    G->kernels = (int)(ws_kernel_launches() - launches0);
    countLaunch(-G->kernels);  // captured, not launched
    restore();
    WS_CK(cudaStreamDestroy(cs));
    *out = G.release();
  });
}

int ws_exec_group_run(ws_exec_group* G, const ws_expr_env* const* envs) {
  return guardedCall([&] {
    if (!envs) throw Error("exec group: no constants", WS_ERR_ARG);
    for (size_t i = 0; i < G->xs.size(); ++i)
      if (!envs[i] || codeDigest(*envs[i]) != G->xs[i]->code)
        throw Error("exec group: query " + std::to_string(i) + "'s expressions differ from its prepared query's",
                    WS_ERR_ARG);
    // the previous run's graph copies `stage` when it runs: wait for it before overwriting
    WS_CK(cudaEventSynchronize(G->done));
    for (size_t j = 0; j < G->mp.live.size(); ++j) {
      Launch L = G->mp.L[j];
      L.env = envK(*envs[(size_t)G->mp.live[j]]);
      memcpy(G->stage + j * sizeof(Launch), &L, sizeof(Launch));
    }
    WS_CK(cudaGraphLaunch(G->exec, stream()));
    WS_CK(cudaEventRecord(G->done, stream()));
    countLaunch(G->kernels);
  });
}

void ws_exec_group_destroy(ws_exec_group* G) { delete G; }

int ws_host_alloc(size_t bytes, void** out) {
  return guardedCall([&] {
    *out = nullptr;
    ws_gpu_init();
    if (cudaHostAlloc(out, std::max<size_t>(bytes, 1), cudaHostAllocMapped) != cudaSuccess) {
      cudaGetLastError();
      *out = nullptr;
      throw Error("pinned host allocation of " + std::to_string(bytes) + " bytes failed", WS_ERR_OOM);
    }
  });
}

int ws_host_free(void* p) {
  return guardedCall([&] {
    if (p) WS_CK(cudaFreeHost(p));
  });
}

int ws_agg_sum_bits_slots(const ws_aggregator* A, uint8_t* out) {
  for (int a = 0; a < A->plan.naggs; ++a) {
    if (A->plan.nkeys) out[a] = A->plan.aggBits[a];
    else
      out[a] = (A->plan.ops[a] == WS_AGG_SUM || A->plan.ops[a] == WS_AGG_MIN || A->plan.ops[a] == WS_AGG_MAX) && A->plan.aggInt[a];
  }
  return WS_OK;
}

int ws_agg_sum_high(const ws_aggregator* A, int64_t* out) {
  for (int a = 0; a < A->plan.naggs; ++a) out[a] = a < (int)A->hi.size() ? A->hi[a] : 0;
  return WS_OK;
}

int ws_agg_compact(ws_aggregator* A, double** keys, double** accs, int64_t* ngroups) {
  return guardedCall([&] {
    checkFlags(*A, nullptr);
    const int nk = A->plan.nkeys, na = A->plan.naggs;
    DBuf<int64_t> idx;
    const int64_t g = nk ? aggCompactIdx(*A, idx) : 1;
    DBuf<double> dk(std::max<int64_t>(g * nk, 1)), da(std::max<int64_t>(g * na, 1));
    DBuf<int64_t> dx(std::max<int64_t>(g * na * 2, 1));
    DBuf<int16_t> pk(WS_MAX_AGGS);
    if (g) {
      WS_LAUNCH(kEmit, gridFor(g), 256, 0, A->rows.p, nk ? idx.p : nullptr, g, emitSpec(*A), dk.p, dx.p, 1);
      int16_t* st = (int16_t*)pinnedStage(2 * WS_MAX_AGGS);
      for (int a = 0; a < WS_MAX_AGGS; ++a) st[a] = a < na ? A->lay.kind[A->lay.partner[a]] : 0;
      h2dAsync(pk.p, st, 2 * WS_MAX_AGGS);
      stageCopied();
      WS_LAUNCH(kExactToDouble, gridFor(g), 256, 0, dx.p, g, dblSpec(*A), pk.p, da.p, 1);
    }
    *keys = dk.release();
    *accs = da.release();
    *ngroups = g;
  });
}

}  // extern "C"
