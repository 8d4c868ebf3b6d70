// Relational helpers around the scan / join operators: join-filter key bitmaps and deleted bits,
// dictionary code remaps, NULL-aware and encoded gathers, expression evaluation at row indices
// (projection and post-aggregation keys), and the stable multi-key sort permutation of ORDER BY
// (reference: src/gpu.cu:149-163, :802-888, :1011-1087, :1323-1367).
#include <climits>
#include <cmath>
#include <cstring>

#include "ws_internal.h"
#include "ws_interp.cuh"

namespace ws {
namespace {

int gridFor(int64_t n, int block = 256, int perSm = 8) {
  int64_t g = (n + block - 1) / block;
  const int64_t cap = (int64_t)smCount() * perSm;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}
#define WS_LAUNCH(kernel, grid, block, smem, ...)               \
  do {                                                          \
    kernel<<<(grid), (block), (smem), stream()>>>(__VA_ARGS__); \
    WS_CK(cudaGetLastError());                                  \
    countLaunch();                                              \
  } while (0)
#define WS_GRID_STRIDE(j, n) \
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < (n); j += (int64_t)gridDim.x * blockDim.x)

// ---------------------------------------------------------------- bitmaps, codes, gathers
// Join-key values are read like the join's keys: I32 widened, I64 as stored, F64 truncated; the
// NULL sentinels / NaN never set a bit.
__device__ __forceinline__ bool keyOf(const ws_col_view& c, int64_t r, long long& k) {
  if (c.t == 0 || c.t == 3) {
    const int v = ((const int*)c.p)[r];
    k = v;
    return v != WS_NULL_I32;
  }
  if (c.t == 1 || c.t == 4) {
    k = ((const long long*)c.p)[r];
    return k != WS_NULL_I64;
  }
  const double d = ((const double*)c.p)[r];
  k = (long long)d;
  return d == d;
}

__global__ void kKeyBitmap(ws_col_view key, int64_t n, long long lo, int64_t nbits, uint32_t* bits) {
  WS_GRID_STRIDE(i, n) {
    long long k;
    if (!keyOf(key, i, k)) continue;
    const u64 v = (u64)k - (u64)lo;
    if (v < (u64)nbits) atomicOr(bits + (v >> 5), 1u << (v & 31));
  }
}
__global__ void kSetBits(uint32_t* bits, const int32_t* idx, int64_t m) {
  WS_GRID_STRIDE(j, m) atomicOr(bits + (idx[j] >> 5), 1u << (idx[j] & 31));
}
__global__ void kRemapCodes(const int32_t* in, int64_t n, const int32_t* map, int64_t mapN, int32_t* out) {
  WS_GRID_STRIDE(j, n) {
    const int32_t c = in[j];
    out[j] = c == WS_NULL_I32 ? WS_NULL_I32 : (c >= 0 && c < mapN) ? __ldg(map + c) : -2;
  }
}
__global__ void kBitsToDouble(const double* src, int64_t n, double* dst) {
  WS_GRID_STRIDE(j, n) dst[j] = (double)__double_as_longlong(src[j]);
}
template <class T>
__global__ void kGatherNull(const T* src, const int32_t* idx, int64_t m, T* dst, T nul) {
  WS_GRID_STRIDE(j, m) dst[j] = idx[j] < 0 ? nul : src[idx[j]];
}
// fixed-size elements of `words` 32-bit words; index -1 gives a NULL element (NaN floats when nulls,
// else zeros)
__global__ void kGatherWords(const uint32_t* src, int words, const int32_t* idx, int64_t m, uint32_t* dst, int nulls) {
  WS_GRID_STRIDE(j, m * words) {
    const int64_t r = j / words, w = j % words;
    const int32_t i = idx[r];
    dst[j] = i < 0 ? (nulls ? 0x7fc00000u : 0u) : src[(int64_t)i * words + w];
  }
}
// encoded segment column -> raw values (NULL sentinels kept as stored for integers)
__global__ void kGatherEnc(ws_col_view v, int ptype, const int32_t* idx, int64_t m, void* dst) {
  WS_GRID_STRIDE(j, m) {
    const i64 r = idx[j];
    if (ptype == WS_PT_F64) ((double*)dst)[j] = colDblAt(v, r);
    else if (ptype == WS_PT_I32) ((int32_t*)dst)[j] = (int32_t)colIntAt(v, r);
    else ((int64_t*)dst)[j] = colIntAt(v, r);
  }
}

// ---------------------------------------------------------------- evaluation at rows
struct EvalSpec {
  const TInstr* code;
  int start, len;
  int isInt;                // the program's result type
  int single;               // the program is one integer OP_COL (read exactly)
  int col;
};
// out[j] = the program at row idx[j] (or j): doubles (NULL = NaN) ...
__global__ void kEvalAt(const __grid_constant__ EvalSpec s, const ws_col_view* cv, const __grid_constant__ EnvK env,
                        const int32_t* idx, int64_t m, double* out) {
  WS_GRID_STRIDE(j, m) {
    const Word w = vmRun(s.code, s.start, s.len, cv, idx ? idx[j] : j, env);
    out[j] = s.isInt ? (double)w.i : w.d;
  }
}
// ... or int64 (NULL = the BIGINT NULL sentinel): exact for integer programs, else the double rounded
__global__ void kEvalAtInt(const __grid_constant__ EvalSpec s, const ws_col_view* cv, const __grid_constant__ EnvK env,
                           const int32_t* idx, int64_t m, int64_t* out) {
  WS_GRID_STRIDE(j, m) {
    const i64 r = idx ? idx[j] : j;
    if (s.single) {
      const ws_col_view& c = cv[s.col];
      const i64 v = colIntAt(c, r);
      out[j] = (c.t == 0 || c.t == 3) && v == (i64)WS_NULL_I32 ? (i64)WS_NULL_I64 : v;
      continue;
    }
    const Word w = vmRun(s.code, s.start, s.len, cv, r, env);
    if (s.isInt) out[j] = w.i;
    else out[j] = w.d != w.d ? (i64)WS_NULL_I64 : llround(w.d);
  }
}

// ---------------------------------------------------------------- sort permutation
// Stable LSD radix sort of (64-bit key, int32 permutation) pairs by 4-bit digits: per pass a count
// of each digit per block, one exclusive scan of the counts in digit-major order (the base of every
// (digit, block)), and a scatter in which each block ranks its items in their original order (a scan
// over [digit][thread] counts), so equal keys keep their relative order.  Passes whose digit is the
// same for every item are skipped (a histogram of all 16 digits first).
constexpr int kRThreads = 256, kRItems = 8, kRTile = kRThreads * kRItems, kRBuckets = 16;

// double sort key -> unsigned order key: NULL (NaN) sorts first as -inf, -0 as 0; descending inverts
__device__ __forceinline__ u64 orderKey(double v, bool desc) {
  if (v != v) v = -__longlong_as_double(0x7ff0000000000000ll);
  if (v == 0.0) v = 0.0;
  u64 b = (u64)__double_as_longlong(v);
  b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
  return desc ? ~b : b;
}
__global__ void kSortKeys(const int32_t* perm, const double* key, int64_t m, int desc, u64* out) {
  WS_GRID_STRIDE(j, m) out[j] = orderKey(key[perm ? perm[j] : j], desc != 0);
}
__global__ void kIota(int32_t* p, int64_t m) {
  WS_GRID_STRIDE(j, m) p[j] = (int32_t)j;
}
// hist[d * 16 + v]: items whose digit d (bits 4d..4d+3) is v
__global__ void kDigitHist(const u64* keys, int64_t m, unsigned long long* hist) {
  __shared__ unsigned h[16 * kRBuckets];
  for (int i = threadIdx.x; i < 16 * kRBuckets; i += blockDim.x) h[i] = 0;
  __syncthreads();
  WS_GRID_STRIDE(j, m) {
    const u64 k = keys[j];
#pragma unroll
    for (int d = 0; d < 16; ++d) atomicAdd(&h[d * kRBuckets + ((k >> (4 * d)) & 15)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 16 * kRBuckets; i += blockDim.x)
    if (h[i]) atomicAdd(hist + i, (unsigned long long)h[i]);
}
// counts[v * nblocks + block]: items of the block's tile with digit value v
__global__ void kRadixCount(const u64* keys, int64_t m, int shift, int64_t nblocks, int64_t* counts) {
  __shared__ int h[kRBuckets];
  if (threadIdx.x < kRBuckets) h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRTile;
  for (int i = threadIdx.x; i < kRTile; i += kRThreads) {
    const int64_t j = base + i;
    if (j < m) atomicAdd(&h[(keys[j] >> shift) & 15], 1);
  }
  __syncthreads();
  if (threadIdx.x < kRBuckets) counts[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}
// exclusive scan in place of n counts with one block (total in counts[n])
__global__ void kScanOne(int64_t* counts, int64_t n) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int64_t per = (n + T - 1) / T;
  const int64_t lo = min((int64_t)t * per, n), hi = min(lo + per, n);
  int64_t s = 0;
  for (int64_t i = lo; i < hi; ++i) s += counts[i];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
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
// stable scatter: thread t owns items [t * kRItems, (t + 1) * kRItems) of the tile (in order)
__global__ void kRadixScatter(const u64* keys, const int32_t* vals, int64_t m, int shift, int64_t nblocks,
                              const int64_t* offs, u64* keysOut, int32_t* valsOut) {
  __shared__ int cnt[kRBuckets * kRThreads];  // [digit][thread], then the exclusive scan of it
  __shared__ int wtot[kRThreads / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * kRTile + (int64_t)t * kRItems;
  u64 k[kRItems];
  int32_t v[kRItems];
  int dg[kRItems];
  for (int b = 0; b < kRBuckets; ++b) cnt[b * kRThreads + t] = 0;
#pragma unroll
  for (int i = 0; i < kRItems; ++i) {
    const bool ok = i0 + i < m;
    k[i] = ok ? keys[i0 + i] : 0;
    v[i] = ok ? vals[i0 + i] : 0;
    dg[i] = ok ? (int)((k[i] >> shift) & 15) : -1;
    if (ok) ++cnt[dg[i] * kRThreads + t];
  }
  __syncthreads();
  // exclusive scan over the [digit][thread] counts: thread t scans entries [t * 16, t * 16 + 16)
  int loc[kRBuckets], run = 0;
#pragma unroll
  for (int e = 0; e < kRBuckets; ++e) {
    loc[e] = run;
    run += cnt[t * kRBuckets + e];
  }
  int incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wtot[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wtot[w];
  const int excl = before + incl - run;
  __syncthreads();
#pragma unroll
  for (int e = 0; e < kRBuckets; ++e) cnt[t * kRBuckets + e] = excl + loc[e];
  __syncthreads();
  // cnt[d * kRThreads + t] = items of digit < d in the tile + items of digit d in threads < t
  int bucketStart[kRBuckets];
#pragma unroll
  for (int d = 0; d < kRBuckets; ++d) bucketStart[d] = cnt[d * kRThreads];
  int pos[kRBuckets];
#pragma unroll
  for (int d = 0; d < kRBuckets; ++d) pos[d] = cnt[d * kRThreads + t] - bucketStart[d];
#pragma unroll
  for (int i = 0; i < kRItems; ++i) {
    if (dg[i] < 0) continue;
    int p = 0;
#pragma unroll
    for (int d = 0; d < kRBuckets; ++d)
      if (d == dg[i]) p = pos[d]++;
    const int64_t at = offs[(int64_t)dg[i] * nblocks + blockIdx.x] + p;
    keysOut[at] = k[i];
    valsOut[at] = v[i];
  }
}
__global__ void kMapRank(double* keys, const int32_t* rank, int64_t m) {
  WS_GRID_STRIDE(j, m) keys[j] = keys[j] != keys[j] ? -1.0 : (double)__ldg(rank + (int64_t)keys[j]);
}

// ---------------------------------------------------------------- distinct values, bitmaps, temp columns
// bit (v - base) of every non-NULL value v in [base, base + span) of an exact int64 array
__global__ void kDistinctBits(const i64* v, int64_t m, i64 base, i64 span, uint32_t* bits) {
  WS_GRID_STRIDE(j, m) {
    const i64 x = v[j];
    if (x == (i64)WS_NULL_I64) continue;
    const u64 k = (u64)x - (u64)base;
    if ((i64)k < 0 || (i64)k >= span || x < base) continue;
    const uint32_t bit = 1u << (k & 31);
    if (!(__ldg(bits + (k >> 5)) & bit)) atomicOr(bits + (k >> 5), bit);
  }
}
// bit (v - base) of the non-NULL values of an INT (out 0) / BIGINT (out 1) column; *nul: any NULL
__global__ void kBitsFromColumn(const void* col, int out, int64_t n, i64 base, i64 nbits, uint32_t* bits, int* nul) {
  int sawNull = 0;
  WS_GRID_STRIDE(i, n) {
    i64 v;
    if (out == 1) {
      v = ((const i64*)col)[i];
      if (v == (i64)WS_NULL_I64) {
        sawNull = 1;
        continue;
      }
    } else {
      const int x = ((const int*)col)[i];
      if (x == WS_NULL_I32) {
        sawNull = 1;
        continue;
      }
      v = x;
    }
    const i64 k = v - base;
    if (k >= 0 && k < nbits) atomicOr(bits + (k >> 5), 1u << (k & 31));
  }
  if (__any_sync(0xffffffffu, sawNull) && (threadIdx.x & 31) == 0) atomicOr(nul, 1);
}
// One temp-table column from compacted groups (column-major keys / accs); min / max of an integer
// output over the non-NULL groups (mnmx[0] / [1]).
__global__ void kTempColumn(const double* keys, const double* accs, int64_t g, const __grid_constant__ ws_temp_col_spec s,
                            void* out, long long* mnmx) {
  long long mn = LLONG_MAX, mx = LLONG_MIN;
  WS_GRID_STRIDE(r, g) {
    auto A = [&](int j) { return accs[(int64_t)j * g + r]; };
    auto bits = [](double d) { return (i64)__double_as_longlong(d); };
    bool nul = s.src == 1 && s.cnt >= 0 && A(s.cnt) == 0;
    bool isInt = false;
    i64 iv = 0;
    double dv = 0;
    if (s.src == 0) {
      const double k = keys[(int64_t)s.idx * g + r];
      if (s.key_int) {
        iv = bits(k);
        isInt = true;
        nul = iv == (i64)WS_NULL_I64 || iv == (i64)WS_NULL_I32;
      } else {
        dv = k;
        nul = k != k;
      }
    } else if (!nul) {
      switch (s.kind) {
        case 1: iv = bits(A(s.idx)); isInt = true; break;
        case 2: iv = (i64)((u64)bits(A(s.hi)) * 4294967296ull + (u64)bits(A(s.idx))); isInt = true; break;
        case 3: iv = (i64)A(s.idx); isInt = true; break;
        case 4: {
          const double sum = s.sum_bits ? (s.hi >= 0 ? (double)bits(A(s.hi)) * 4294967296.0 + (double)bits(A(s.idx))
                                                     : (double)bits(A(s.idx)))
                                        : A(s.idx);
          dv = sum / s.div / A(s.cnt);
          break;
        }
        default:
          dv = A(s.idx) / s.div;
          nul = dv != dv;
      }
    }
    if (s.mul != 1 && !nul) {
      dv = (isInt ? (double)iv : dv) * s.mul;
      isInt = false;
    }
    if (s.out == 2) {
      ((double*)out)[r] = nul ? __longlong_as_double(0x7ff8000000000000ll) : isInt ? (double)iv : dv;
      continue;
    }
    const long long v = nul ? 0 : isInt ? iv : llround(dv);
    if (!nul) mn = v < mn ? v : mn, mx = v > mx ? v : mx;
    if (s.out == 1) ((i64*)out)[r] = nul ? (i64)WS_NULL_I64 : v;
    else ((int32_t*)out)[r] = nul ? WS_NULL_I32 : (int32_t)v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const long long a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
  if ((threadIdx.x & 31) == 0 && mn <= mx) {
    atomicMin(&mnmx[0], mn);
    atomicMax(&mnmx[1], mx);
  }
}
// host column of ptype -> double sort keys
__global__ void kToDouble(const void* src, int ptype, int64_t n, double* out) {
  WS_GRID_STRIDE(i, n) {
    out[i] = ptype == WS_PT_I32 ? (double)((const int*)src)[i]
             : ptype == WS_PT_I64 ? (double)((const i64*)src)[i] : ((const double*)src)[i];
  }
}

// The engine evaluates gpuDistinctInts' program exactly only when it is built of integer columns,
// integer literals, + - * and negation within a 16-deep stack (src/gpu.cu:826-865); any other program
// yields no values.
bool exactIntProgram(const ws_expr_env& env, ws_prog p) {
  int sp = 0;
  for (int i = 0; i < p.len; ++i) {
    const ws_instr in = env.code[p.start + i];
    switch (in.op) {
      case WS_OP_COL: {
        const int t = env.cols[in.arg].t;
        if (t == 2 || t == 5 || t == 6 || sp >= 16) return false;
        ++sp;
        break;
      }
      case WS_OP_CONST:
        if (!in.isInt || sp >= 16) return false;
        ++sp;
        break;
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL:
        if (sp < 2) return false;
        --sp;
        break;
      case WS_OP_NEG:
        if (sp < 1) return false;
        break;
      default: return false;
    }
  }
  return sp == 1;
}

double kNullF64() {  // the engine's NULL double: the canonical quiet NaN
  const uint64_t b = 0x7ff8000000000000ull;
  double d;
  memcpy(&d, &b, 8);
  return d;
}

EvalSpec evalSpec(const ws_expr_env& env, int ncols, ws_prog prog, DBuf<uint8_t>& progBuf) {
  if (ncols < 0 || ncols > WS_MAX_COLS) throw Error("bad column count", WS_ERR_ARG);
  ws_agg_plan plan;
  memset(&plan, 0, sizeof plan);
  plan.hasWhere = 1;
  plan.where = prog;
  plan.naggs = 1;  // the hidden COUNT(*) slot only (no program): the layout needs one slot
  plan.ops[0] = WS_AGG_COUNT;
  TProgs* tp = new TProgs;
  try {
    buildTProgs(env, ncols, plan, true, *tp);
  } catch (...) {
    delete tp;
    throw;
  }
  EvalSpec s{};
  s.start = tp->where[0];
  s.len = tp->where[1];
  s.isInt = typeProg(env, prog, ncols).isInt() ? 1 : 0;
  const ws_instr& in0 = env.code[prog.start];
  s.single = prog.len == 1 && in0.op == WS_OP_COL && env.cols[in0.arg].t != 2 ? 1 : 0;
  s.col = in0.arg;
  const size_t bytes = sizeof(TInstr) * (size_t)std::max(s.start + s.len, 1);
  progBuf = DBuf<uint8_t>((int64_t)bytes);
  uint8_t* st = pinnedStage(bytes);
  memcpy(st, tp->code, bytes);
  delete tp;
  h2dAsync(progBuf.p, st, bytes);
  stageCopied();
  s.code = (const TInstr*)progBuf.p;
  return s;
}

const ws_col_view* uploadCols(const ws_expr_env& env, int ncols, DBuf<uint8_t>& buf) {
  if (ncols < 0 || ncols > WS_MAX_COLS) throw Error("bad column count", WS_ERR_ARG);
  const size_t bytes = sizeof(ws_col_view) * (size_t)std::max(ncols, 1);
  buf = DBuf<uint8_t>((int64_t)bytes);
  uint8_t* st = pinnedStage(bytes);
  memcpy(st, env.cols, sizeof(ws_col_view) * (size_t)ncols);
  h2dAsync(buf.p, st, bytes);
  stageCopied();
  return (const ws_col_view*)buf.p;
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

int ws_key_bitmap(ws_col_view key, int64_t n, int64_t lo, int64_t nbits, uint32_t* bits) {
  return guardedCall([&] {
    if (nbits < 0) throw Error("negative bitmap size", WS_ERR_ARG);
    WS_CK(cudaMemsetAsync(bits, 0, (size_t)((nbits + 31) / 32) * 4, stream()));
    if (n > 0 && nbits > 0) WS_LAUNCH(kKeyBitmap, gridFor(n), 256, 0, key, n, (long long)lo, nbits, bits);
  });
}

int ws_set_bits(uint32_t* bits, const int32_t* idx, int64_t m) {
  return guardedCall([&] {
    if (m > 0) WS_LAUNCH(kSetBits, gridFor(m), 256, 0, bits, idx, m);
  });
}

int ws_remap_codes(const int32_t* in, int64_t n, const int32_t* map, int64_t map_n, int32_t* out) {
  return guardedCall([&] {
    if (n > 0) WS_LAUNCH(kRemapCodes, gridFor(n), 256, 0, in, n, map, map_n, out);
  });
}

int ws_bits_to_double(const double* src, int64_t n, double* dst) {
  return guardedCall([&] {
    if (n > 0) WS_LAUNCH(kBitsToDouble, gridFor(n), 256, 0, src, n, dst);
  });
}

int ws_gather_null(const void* src, int ptype, const int32_t* idx, int64_t m, void* dst) {
  return guardedCall([&] {
    if (m <= 0) return;
    if (ptype == WS_PT_I32)
      WS_LAUNCH(kGatherNull<int32_t>, gridFor(m), 256, 0, (const int32_t*)src, idx, m, (int32_t*)dst, (int32_t)WS_NULL_I32);
    else if (ptype == WS_PT_I64)
      WS_LAUNCH(kGatherNull<long long>, gridFor(m), 256, 0, (const long long*)src, idx, m, (long long*)dst,
                (long long)WS_NULL_I64);
    else if (ptype == WS_PT_F64)
      WS_LAUNCH(kGatherNull<double>, gridFor(m), 256, 0, (const double*)src, idx, m, (double*)dst, kNullF64());
    else
      throw Error("gather: unsupported physical type", WS_ERR_ARG);
  });
}

int ws_gather_bytes(const void* src, int esize, const int32_t* idx, int64_t m, void* dst, int nulls) {
  return guardedCall([&] {
    if (esize <= 0 || esize % 4) throw Error("gather: element size must be a multiple of 4 bytes", WS_ERR_ARG);
    if (m > 0) WS_LAUNCH(kGatherWords, gridFor(m * (esize / 4)), 256, 0, (const uint32_t*)src, esize / 4, idx, m,
                         (uint32_t*)dst, nulls);
  });
}

int ws_gather_enc(ws_col_view v, int ptype, const int32_t* idx, int64_t m, void* dst) {
  return guardedCall([&] {
    if (m <= 0) return;
    ws_col_view w = v;
    w.t = ptype == WS_PT_I32 ? 3 : ptype == WS_PT_I64 ? 4 : 2;  // NULL sentinels kept as stored
    WS_LAUNCH(kGatherEnc, gridFor(m), 256, 0, w, ptype, idx, m, dst);
  });
}

int ws_eval_at(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, double* out) {
  return guardedCall([&] {
    if (m <= 0) return;
    DBuf<uint8_t> pb, cb;
    const EvalSpec s = evalSpec(*env, ncols, prog, pb);
    const ws_col_view* cv = uploadCols(*env, ncols, cb);
    WS_LAUNCH(kEvalAt, gridFor(m), 256, 0, s, cv, envK(*env), idx, m, out);
  });
}

int ws_eval_at_int(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, int64_t* out) {
  return guardedCall([&] {
    if (m <= 0) return;
    DBuf<uint8_t> pb, cb;
    const EvalSpec s = evalSpec(*env, ncols, prog, pb);
    const ws_col_view* cv = uploadCols(*env, ncols, cb);
    WS_LAUNCH(kEvalAtInt, gridFor(m), 256, 0, s, cv, envK(*env), idx, m, out);
  });
}

int ws_sort_perm(const double* const* keys, const int* desc, int nkeys, int64_t m, int32_t** out_perm) {
  return guardedCall([&] {
    *out_perm = nullptr;
    if (m < 0 || m > INT32_MAX) throw Error("sort: row count out of range", WS_ERR_ARG);
    DBuf<int32_t> perm(std::max<int64_t>(m, 1)), perm2(std::max<int64_t>(m, 1));
    if (m > 0) {
      WS_LAUNCH(kIota, gridFor(m), 256, 0, perm.p, m);
      DBuf<u64> k1(m), k2(m);
      const int64_t nblocks = (m + kRTile - 1) / kRTile;
      DBuf<int64_t> counts(kRBuckets * nblocks + 1);
      DBuf<unsigned long long> hist(16 * kRBuckets);
      std::vector<unsigned long long> h(16 * kRBuckets);
      for (int key = nkeys - 1; key >= 0; --key) {  // least significant key first (LSD over keys too)
        WS_LAUNCH(kSortKeys, gridFor(m), 256, 0, perm.p, keys[key], m, desc[key], k1.p);
        WS_CK(cudaMemsetAsync(hist.p, 0, 8 * h.size(), stream()));
        WS_LAUNCH(kDigitHist, gridFor(m), 256, 0, k1.p, m, hist.p);
        d2hSync(h.data(), hist.p, 8 * h.size());
        for (int d = 0; d < 16; ++d) {
          bool trivial = false;
          for (int v = 0; v < kRBuckets; ++v) trivial |= h[d * kRBuckets + v] == (unsigned long long)m;
          if (trivial) continue;  // every item has the same digit: the pass would not move anything
          WS_LAUNCH(kRadixCount, (unsigned)nblocks, kRThreads, 0, k1.p, m, 4 * d, nblocks, counts.p);
          WS_LAUNCH(kScanOne, 1, 1024, 0, counts.p, kRBuckets * nblocks);
          WS_LAUNCH(kRadixScatter, (unsigned)nblocks, kRThreads, 0, k1.p, perm.p, m, 4 * d, nblocks, counts.p, k2.p,
                    perm2.p);
          std::swap(k1, k2);
          std::swap(perm, perm2);
        }
      }
    }
    *out_perm = perm.release();
  });
}

int ws_distinct_ints(const ws_expr_env* env, int ncols, ws_prog prog, const int32_t* idx, int64_t m, int64_t base,
                     int64_t span, int64_t* out, int64_t max_out, int64_t* count) {
  return guardedCall([&] {
    *count = 0;
    if (m <= 0 || span <= 0) return;
    if (prog.start < 0 || prog.len <= 0 || prog.start + prog.len > WS_MAX_CODE)
      throw Error("ws_distinct_ints: program outside the code array", WS_ERR_ARG);
    if (!exactIntProgram(*env, prog)) return;
    if (span > ((int64_t)1 << 40)) throw Error("ws_distinct_ints: span too large for a bitmap", WS_ERR_ARG);
    DBuf<uint8_t> pb, cb;
    const EvalSpec s = evalSpec(*env, ncols, prog, pb);
    const ws_col_view* cv = uploadCols(*env, ncols, cb);
    DBuf<i64> vals(m);
    WS_LAUNCH(kEvalAtInt, gridFor(m), 256, 0, s, cv, envK(*env), idx, m, (int64_t*)vals.p);
    const int64_t words = (span + 31) / 32;
    DBuf<uint32_t> bits(words);
    WS_CK(cudaMemsetAsync(bits.p, 0, (size_t)words * 4, stream()));
    WS_LAUNCH(kDistinctBits, gridFor(m), 256, 0, vals.p, m, base, span, bits.p);
    std::vector<uint32_t> h((size_t)words);
    d2hLarge(h.data(), bits.p, (size_t)words * 4);
    int64_t c = 0;
    for (int64_t w = 0; w < words; ++w)
      for (uint32_t b = h[(size_t)w]; b; b &= b - 1) {
        if (c < max_out && out) out[c] = base + w * 32 + __builtin_ctz(b);
        ++c;
      }
    *count = c;
    if (c > max_out) throw Error("ws_distinct_ints: more distinct values than out holds", WS_ERR_SIZE);
  });
}

int ws_bits_from_column(const void* col, int out, int64_t n, int64_t base, int64_t nbits, uint32_t** bits,
                        int* saw_null) {
  return guardedCall([&] {
    ensureInit();
    *bits = nullptr;
    *saw_null = 0;
    if (nbits < 0 || n < 0 || (out != 0 && out != 1)) throw Error("ws_bits_from_column: bad arguments", WS_ERR_ARG);
    const size_t bytes = std::max<size_t>(4, (size_t)((nbits + 31) / 32) * 4);
    uint32_t* b = nullptr;
    WS_CK(cudaMalloc(&b, bytes));
    try {
      WS_CK(cudaMemsetAsync(b, 0, bytes, stream()));
      DBuf<int> nul(1);
      WS_CK(cudaMemsetAsync(nul.p, 0, 4, stream()));
      if (n > 0) WS_LAUNCH(kBitsFromColumn, gridFor(n), 256, 0, col, out, n, base, nbits, b, nul.p);
      int h = 0;
      d2hSync(&h, nul.p, 4);
      *saw_null = h != 0;
    } catch (...) {
      cudaStreamSynchronize(stream());
      cudaFree(b);
      throw;
    }
    *bits = b;
  });
}

int ws_temp_column(const double* keys, int nk, const double* accs, int na, int64_t g, const ws_temp_col_spec* s,
                   void** col, double* mn, double* mx) {
  return guardedCall([&] {
    ensureInit();
    *col = nullptr;
    if (g < 0 || s->out > 2 || (s->src == 0 && (s->idx < 0 || s->idx >= nk)) ||
        (s->src == 1 && (s->idx < 0 || s->idx >= na || s->hi >= na || s->cnt >= na)))
      throw Error("ws_temp_column: spec outside the groups' keys / slots", WS_ERR_ARG);
    const size_t w = s->out == 0 ? 4 : 8;
    void* o = nullptr;
    WS_CK(cudaMalloc(&o, std::max<size_t>(1, (size_t)g * w)));
    long long h[2] = {LLONG_MAX, LLONG_MIN};
    try {
      DBuf<long long> mm(2);
      uint8_t* st = pinnedStage(sizeof h);
      memcpy(st, h, sizeof h);
      h2dAsync(mm.p, st, sizeof h);
      stageCopied();
      if (g > 0) WS_LAUNCH(kTempColumn, gridFor(g), 256, 0, keys, accs, g, *s, o, mm.p);
      d2hSync(h, mm.p, sizeof h);
    } catch (...) {
      cudaStreamSynchronize(stream());
      cudaFree(o);
      throw;
    }
    *mn = s->out == 2 || h[0] > h[1] ? -INFINITY : (double)h[0];
    *mx = s->out == 2 || h[0] > h[1] ? INFINITY : (double)h[1];
    *col = o;
  });
}

int ws_sort_perm_host(const void* host_col, int ptype, int64_t n, int32_t* perm) {
  return guardedCall([&] {
    if (n <= 0) return;
    if (ptype != WS_PT_I32 && ptype != WS_PT_I64 && ptype != WS_PT_F64)
      throw Error("ws_sort_perm_host: ptype must be I32, I64 or F64", WS_ERR_ARG);
    const size_t esz = ptype == WS_PT_I32 ? 4 : 8;
    DBuf<uint8_t> raw((int64_t)(n * esz));
    WS_CK(cudaMemcpyAsync(raw.p, host_col, (size_t)n * esz, cudaMemcpyHostToDevice, stream()));
    DBuf<double> k(n);
    WS_LAUNCH(kToDouble, gridFor(n), 256, 0, raw.p, ptype, n, k.p);
    const double* keys[1] = {k.p};
    const int desc[1] = {0};
    int32_t* p = nullptr;
    const int rc = ws_sort_perm(keys, desc, 1, n, &p);
    if (rc != WS_OK) throw Error(ws_last_error(), rc);
    DBuf<int32_t> pp;
    pp.p = p, pp.n = n;
    d2hLarge(perm, p, (size_t)n * 4);
  });
}

int ws_map_rank(double* keys, const int32_t* rank, int64_t m) {
  return guardedCall([&] {
    if (m > 0) WS_LAUNCH(kMapRank, gridFor(m), 256, 0, keys, rank, m);
  });
}

}  // extern "C"
