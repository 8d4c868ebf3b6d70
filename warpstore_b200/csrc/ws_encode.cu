// Segment encoding on the GPU (the flush path of the engine's storage: src/storage.cu:1138-1192 encodes
// segment columns on the host): integer columns to the bit-packed (enc 7) or run-length (enc 8)
// formats that the scan kernels decode (formats: ws_dev.cuh), and any column to the engine's own
// formats by the engine's rule (ws_encode_column_engine: frame of reference, dictionary, decimal).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "ws_internal.h"

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

__device__ __forceinline__ long long rawAt(const void* src, int i32, int64_t i) {
  return i32 ? (long long)((const int*)src)[i] : ((const long long*)src)[i];
}

// st[0] = min, st[1] = max of the non-NULL values, st[2] = any NULL
__global__ void kMinMax(const void* src, int i32, long long nul, int64_t n, long long* st) {
  long long mn = 0x7fffffffffffffffll, mx = (long long)0x8000000000000000ull;
  int anyNull = 0;
  WS_GRID_STRIDE(i, n) {
    const long long v = rawAt(src, i32, i);
    if (v == nul) anyNull = 1;
    else mn = min(mn, v), mx = max(mx, v);
  }
  for (int o = 16; o; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    anyNull |= __shfl_xor_sync(0xffffffffu, anyNull, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(st, mn);
    atomicMax(st + 1, mx);
    if (anyNull) atomicOr((int*)(st + 2), 1);
  }
}

// bit-packed words: word w holds bits [32w, 32w + 32) of the code stream
__global__ void kPack(const void* src, int i32, long long nul, int64_t n, long long base, int b, int64_t nwords,
                      unsigned* words) {
  const unsigned nulc = b == 32 ? 0xffffffffu : ((1u << b) - 1u);
  WS_GRID_STRIDE(w, nwords) {
    const u64 lo = (u64)w * 32, hi = lo + 32;  // bit range of this word
    unsigned out = 0;
    for (u64 row = lo / (u64)b; row < (u64)n && row * (u64)b < hi; ++row) {
      const long long v = rawAt(src, i32, (int64_t)row);
      const unsigned code = v == nul ? nulc : (unsigned)(v - base);
      const u64 start = row * (u64)b;
      if (start >= lo) out |= code << (start - lo);
      else out |= code >> (lo - start);
    }
    words[w] = out;
  }
}

// run starts: row i starts a run when it is row 0 or differs from row i - 1
__global__ void kRunCount(const void* src, int i32, int64_t n, int64_t* counts) {
  __shared__ int wsum[8];
  const int64_t i0 = (int64_t)blockIdx.x * 1024 + threadIdx.x * 4;
  int c = 0;
  for (int k = 0; k < 4; ++k) {
    const int64_t i = i0 + k;
    c += i < n && (i == 0 || rawAt(src, i32, i) != rawAt(src, i32, i - 1));
  }
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += wsum[w];
    counts[blockIdx.x] = t;
  }
}
__global__ void kScanChunks(int64_t* counts, int64_t n) {  // exclusive scan in place, total in counts[n]
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
// run k: starts[k] = its first row, vals[k] = its value (in order)
__global__ void kRunWrite(const void* src, int i32, int64_t n, const int64_t* offs, int* starts, long long* vals) {
  __shared__ int wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * 1024 + threadIdx.x * 4;
  bool f[4];
  int c = 0;
  for (int k = 0; k < 4; ++k) {
    const int64_t i = i0 + k;
    f[k] = i < n && (i == 0 || rawAt(src, i32, i) != rawAt(src, i32, i - 1));
    c += f[k];
  }
  int incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  int64_t at = offs[blockIdx.x] + before + incl - c;
  for (int k = 0; k < 4; ++k)
    if (f[k]) starts[at] = (int)(i0 + k), vals[at] = rawAt(src, i32, i0 + k), ++at;
}
__global__ void kRunEnds(const int* starts, int64_t runs, int64_t n, int* ends) {
  WS_GRID_STRIDE(k, runs) ends[k] = k + 1 < runs ? starts[k + 1] : (int)n;
}

// ---- the engine's formats (src/storage.cu:1093-1192).  enc 1/2/3: integer offsets from the minimum as
// uint8 / uint16 / uint32 (all-ones = NULL); enc 4: a dictionary of at most 255 distinct doubles (bit
// patterns, in order of first occurrence) and uint8 codes; enc 5/6: doubles that are exact decimals,
// llround(x * 10^s) - minimum as uint16 / uint32 (all-ones = NaN).  Header: int64 base (the minimum),
// double 10^s (enc 5/6); enc 4's 256 dictionary entries follow the header.
__global__ void kEncodeFor(const void* src, int i32, long long nul, int64_t n, long long mn, int w, uint8_t* d) {
  WS_GRID_STRIDE(i, n) {
    const long long v = rawAt(src, i32, i);
    const u64 code = v == nul ? ~0ull : (u64)v - (u64)mn;
    if (w == 1) d[i] = (uint8_t)code;
    else if (w == 2) ((uint16_t*)d)[i] = (uint16_t)code;
    else ((uint32_t*)d)[i] = (uint32_t)code;
  }
}

// Distinct bit patterns of a double column, up to 255 of them: a 4096-slot open-addressing set
// (key 0 = empty; the pattern 0, +0.0, has its own flag) with each pattern's first row (atomicMin).
// Once more than 255 patterns were claimed, *over is set and the threads stop inserting.
constexpr int kDictSlots = 4096;
constexpr long long kFirstNone = 0x7f7f7f7f7f7f7f7fll;  // "no row yet" (the first-row arrays' memset value)
__global__ void kDictInsert(const double* x, int64_t n, u64* keys, long long* first, long long* zeroFirst, int* count,
                            int* over) {
  WS_GRID_STRIDE(i, n) {
    if (*(volatile int*)over) return;
    const u64 b = (u64)__double_as_longlong(x[i]);
    if (b == 0) {
      if (atomicMin(zeroFirst, (long long)i) == kFirstNone && atomicAdd(count, 1) >= 255) *over = 1;
      continue;
    }
    unsigned s = (unsigned)(mix64(b) & (kDictSlots - 1));
    for (int p = 0; p < kDictSlots; ++p) {
      const u64 prev = atomicCAS((unsigned long long*)(keys + s), 0ull, b);
      if (prev == 0ull) {
        if (atomicAdd(count, 1) >= 255) *over = 1;
        atomicMin(first + s, (long long)i);
        break;
      }
      if (prev == b) {
        atomicMin(first + s, (long long)i);
        break;
      }
      s = (s + 1) & (kDictSlots - 1);
    }
  }
}
// codes of the set's patterns (code[slot]; zeroCode for +0.0) -> uint8 codes of the rows
__global__ void kDictEncode(const double* x, int64_t n, const u64* keys, const uint8_t* code, int zeroCode, uint8_t* d) {
  WS_GRID_STRIDE(i, n) {
    const u64 b = (u64)__double_as_longlong(x[i]);
    uint8_t c = (uint8_t)zeroCode;
    if (b != 0) {
      unsigned s = (unsigned)(mix64(b) & (kDictSlots - 1));
      for (int p = 0; p < kDictSlots && keys[s] != b; ++p) s = (s + 1) & (kDictSlots - 1);
      c = code[s];
    }
    d[i] = c;
  }
}

// Decimal doubles: for each scale s = 0..4 (p = 10^s), whether every non-NaN x has |x p| < 4e15 and
// llround(x p) / p == x, and the min / max of llround(x p): st[3s] = not exact, st[3s+1] = min, st[3s+2] = max.
__global__ void kDecimalStats(const double* x, int64_t n, long long* st) {
  int bad[5] = {0, 0, 0, 0, 0};
  long long mn[5], mx[5];
  double p = 1.0;
#pragma unroll
  for (int s = 0; s < 5; ++s) mn[s] = LLONG_MAX, mx[s] = LLONG_MIN;
  WS_GRID_STRIDE(i, n) {
    const double v = x[i];
    if (v != v) continue;
    p = 1.0;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const double y = v * p;
      if (!(fabs(y) < 4e15)) {
        bad[s] = 1;
      } else {
        const long long k = llround(y);
        if ((double)k / p != v) bad[s] = 1;
        mn[s] = min(mn[s], k), mx[s] = max(mx[s], k);
      }
      p *= 10.0;
    }
  }
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    for (int o = 16; o; o >>= 1) {
      bad[s] |= __shfl_xor_sync(0xffffffffu, bad[s], o);
      mn[s] = min(mn[s], __shfl_xor_sync(0xffffffffu, mn[s], o));
      mx[s] = max(mx[s], __shfl_xor_sync(0xffffffffu, mx[s], o));
    }
    if ((threadIdx.x & 31) == 0) {
      if (bad[s]) atomicOr((int*)(st + 3 * s), 1);
      atomicMin(st + 3 * s + 1, mn[s]);
      atomicMax(st + 3 * s + 2, mx[s]);
    }
  }
}
__global__ void kDecimalEncode(const double* x, int64_t n, double p, long long mn, int w, uint8_t* d) {
  WS_GRID_STRIDE(i, n) {
    const double v = x[i];
    const u64 code = v != v ? ~0ull : (u64)(llround(v * p) - mn);
    if (w == 2) ((uint16_t*)d)[i] = (uint16_t)code;
    else ((uint32_t*)d)[i] = (uint32_t)code;
  }
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

int ws_encode_column(const void* src, int t, int64_t n, int enc, void** out, int64_t* bytes, int* enc_used) {
  return guardedCall([&] {
    *out = nullptr;
    *bytes = 0;
    if (!(t == WS_T_I32 || t == WS_T_I64 || t == WS_T_I32N || t == WS_T_I64N))
      throw Error("encode: integer columns only", WS_ERR_ARG);
    if (enc != 0 && enc != 7 && enc != 8) throw Error("encode: enc must be 0 (choose), 7 or 8", WS_ERR_ARG);
    if (n < 0 || n > INT32_MAX) throw Error("encode: segment row count out of range", WS_ERR_ARG);
    const int i32 = t == WS_T_I32 || t == WS_T_I32N;
    const long long nul = i32 ? (long long)WS_NULL_I32 : (long long)WS_NULL_I64;
    // statistics: min / max / NULL and the run count
    DBuf<long long> st(3);
    const long long init[3] = {0x7fffffffffffffffll, (long long)0x8000000000000000ull, 0};
    uint8_t* sg = pinnedStage(sizeof init);
    memcpy(sg, init, sizeof init);
    h2dAsync(st.p, sg, sizeof init);
    stageCopied();
    if (n) WS_LAUNCH(kMinMax, gridFor(n), 256, 0, src, i32, nul, n, st.p);
    const int64_t nchunks = std::max<int64_t>((n + 1023) / 1024, 1);
    DBuf<int64_t> counts(nchunks + 1);
    WS_CK(cudaMemsetAsync(counts.p, 0, 8 * (nchunks + 1), stream()));
    if (n) {
      WS_LAUNCH(kRunCount, (unsigned)nchunks, 256, 0, src, i32, n, counts.p);
      WS_LAUNCH(kScanChunks, 1, 1024, 0, counts.p, nchunks);
    }
    long long hs[3];
    int64_t runs = 0;
    WS_CK(cudaMemcpyAsync(hs, st.p, sizeof hs, cudaMemcpyDeviceToHost, stream()));
    WS_CK(cudaMemcpyAsync(&runs, counts.p + nchunks, 8, cudaMemcpyDeviceToHost, stream()));
    sync();
    const bool anyValue = hs[0] <= hs[1];
    const long long base = anyValue ? hs[0] : 0;
    const unsigned long long range = anyValue ? (unsigned long long)hs[1] - (unsigned long long)hs[0] : 0;
    int b = 1;  // codes 0 .. range, the all-ones code reserved for NULL
    while (b < 64 && (range + 1) >> b) ++b;
    const int64_t nwords = (n * (int64_t)b + 31) / 32;
    const int64_t packBytes = b <= 32 ? WS_ENC_HEADER + 4 * nwords + 16 : INT64_MAX;
    const int64_t rleBytes = WS_ENC_HEADER + ((runs * 4 + 7) & ~7ll) + 8 * runs + 16;
    int use = enc;
    if (use == 0) use = rleBytes < packBytes ? 8 : 7;
    if (use == 7 && b > 32) throw Error("encode: value range too wide to bit-pack (more than 32 bits)", WS_ERR_RANGE);
    const int64_t total = use == 7 ? packBytes : rleBytes;
    DBuf<uint8_t> buf(total);
    WS_CK(cudaMemsetAsync(buf.p, 0, total, stream()));
    uint8_t* hdr = pinnedStage(16);
    memset(hdr, 0, 16);
    if (use == 7) {
      memcpy(hdr, &base, 8);
      memcpy(hdr + 8, &b, 4);
    } else {
      memcpy(hdr, &runs, 8);
    }
    h2dAsync(buf.p, hdr, 16);
    stageCopied();
    if (use == 7) {
      if (nwords) WS_LAUNCH(kPack, gridFor(nwords), 256, 0, src, i32, nul, n, base, b, nwords, (unsigned*)(buf.p + 16));
    } else if (runs) {
      DBuf<int> starts(runs);
      int* ends = (int*)(buf.p + WS_ENC_HEADER);
      long long* vals = (long long*)(buf.p + WS_ENC_HEADER + ((runs * 4 + 7) & ~7ll));
      WS_LAUNCH(kRunWrite, (unsigned)nchunks, 256, 0, src, i32, n, counts.p, starts.p, vals);
      WS_LAUNCH(kRunEnds, gridFor(runs), 256, 0, starts.p, runs, n, ends);
    }
    *out = buf.release();
    *bytes = total;
    if (enc_used) *enc_used = use;
  });
}

int ws_encode_column_engine(const void* src, int ptype, int64_t n, void** out, int64_t* bytes, int* enc_used) {
  return guardedCall([&] {
    *out = nullptr;
    *bytes = 0;
    *enc_used = 0;
    if (ptype != WS_PT_I32 && ptype != WS_PT_I64 && ptype != WS_PT_F64)
      throw Error("encode: ptype must be I32, I64 or F64", WS_ERR_ARG);
    if (n < 0 || n > INT32_MAX) throw Error("encode: segment row count out of range", WS_ERR_ARG);
    if (n < 1024) return;  // the engine keeps short columns raw
    auto finish = [&](DBuf<uint8_t>& buf, int64_t total, int e) {
      *out = buf.release();
      *bytes = total;
      *enc_used = e;
    };
    if (ptype != WS_PT_F64) {  // frame of reference
      const int i32 = ptype == WS_PT_I32;
      const long long nul = i32 ? (long long)WS_NULL_I32 : (long long)WS_NULL_I64;
      DBuf<long long> st(3);
      const long long init[3] = {LLONG_MAX, LLONG_MIN, 0};
      uint8_t* sg = pinnedStage(sizeof init);
      memcpy(sg, init, sizeof init);
      h2dAsync(st.p, sg, sizeof init);
      stageCopied();
      WS_LAUNCH(kMinMax, gridFor(n), 256, 0, src, i32, nul, n, st.p);
      long long hs[3];
      d2hSync(hs, st.p, sizeof hs);
      long long mn = hs[0], mx = hs[1];
      if (mn > mx) mn = mx = 0;  // every value NULL
      const unsigned long long range = (unsigned long long)mx - (unsigned long long)mn;
      const int e = range < 0xFFull ? 1 : range < 0xFFFFull ? 2 : (!i32 && range < 0xFFFFFFFFull) ? 3 : 0;
      if (!e) return;
      const int w = e == 1 ? 1 : e == 2 ? 2 : 4;
      const int64_t total = WS_ENC_HEADER + n * w + 16;
      DBuf<uint8_t> buf(total);
      WS_CK(cudaMemsetAsync(buf.p, 0, total, stream()));
      uint8_t* hdr = pinnedStage(8);
      memcpy(hdr, &mn, 8);
      h2dAsync(buf.p, hdr, 8);
      stageCopied();
      WS_LAUNCH(kEncodeFor, gridFor(n), 256, 0, src, i32, nul, n, mn, w, buf.p + WS_ENC_HEADER);
      finish(buf, total, e);
      return;
    }
    const double* x = (const double*)src;
    // dictionary of at most 255 distinct bit patterns, in order of first occurrence
    {
      DBuf<u64> keys(kDictSlots);
      DBuf<long long> first(kDictSlots + 1);
      DBuf<int> ctl(2);  // [0] count, [1] over
      WS_CK(cudaMemsetAsync(keys.p, 0, 8 * kDictSlots, stream()));
      WS_CK(cudaMemsetAsync(first.p, 0x7f, 8 * (kDictSlots + 1), stream()));  // kFirstNone
      WS_CK(cudaMemsetAsync(ctl.p, 0, 8, stream()));
      WS_LAUNCH(kDictInsert, gridFor(n), 256, 0, x, n, keys.p, first.p, first.p + kDictSlots, ctl.p, ctl.p + 1);
      int hc[2];
      d2hSync(hc, ctl.p, 8);
      if (!hc[1] && hc[0] <= 255) {
        std::vector<u64> hk(kDictSlots);
        std::vector<long long> hf(kDictSlots + 1);
        d2hSync(hk.data(), keys.p, 8 * kDictSlots);
        d2hSync(hf.data(), first.p, 8 * (kDictSlots + 1));
        // entries (first row, slot): slot kDictSlots stands for +0.0
        std::vector<std::pair<long long, int>> ent;
        for (int sl = 0; sl < kDictSlots; ++sl)
          if (hk[(size_t)sl]) ent.push_back({hf[(size_t)sl], sl});
        if (hf[kDictSlots] != kFirstNone) ent.push_back({hf[kDictSlots], kDictSlots});
        std::sort(ent.begin(), ent.end());
        std::vector<uint8_t> code(kDictSlots, 0);
        std::vector<double> vals(256, 0.0);
        int zeroCode = 0;
        for (size_t c = 0; c < ent.size(); ++c) {
          const int sl = ent[c].second;
          if (sl == kDictSlots) {
            zeroCode = (int)c;
            vals[c] = 0.0;
          } else {
            code[(size_t)sl] = (uint8_t)c;
            memcpy(&vals[c], &hk[(size_t)sl], 8);
          }
        }
        const int64_t total = WS_ENC_HEADER + 256 * 8 + n + 16;
        DBuf<uint8_t> buf(total);
        DBuf<uint8_t> dcode(kDictSlots);
        WS_CK(cudaMemsetAsync(buf.p, 0, total, stream()));
        uint8_t* sgv = pinnedStage(256 * 8 + kDictSlots);
        memcpy(sgv, vals.data(), 256 * 8);
        memcpy(sgv + 256 * 8, code.data(), kDictSlots);
        h2dAsync(buf.p + WS_ENC_HEADER, sgv, 256 * 8);
        h2dAsync(dcode.p, sgv + 256 * 8, kDictSlots);
        stageCopied();
        WS_LAUNCH(kDictEncode, gridFor(n), 256, 0, x, n, keys.p, dcode.p, zeroCode, buf.p + WS_ENC_HEADER + 256 * 8);
        finish(buf, total, 4);
        return;
      }
    }
    // decimal doubles: the first scale s at which every value is an exact decimal decides
    DBuf<long long> st(15);
    long long init[15];
    for (int sc = 0; sc < 5; ++sc) init[3 * sc] = 0, init[3 * sc + 1] = LLONG_MAX, init[3 * sc + 2] = LLONG_MIN;
    uint8_t* sg = pinnedStage(sizeof init);
    memcpy(sg, init, sizeof init);
    h2dAsync(st.p, sg, sizeof init);
    stageCopied();
    WS_LAUNCH(kDecimalStats, gridFor(n), 256, 0, x, n, st.p);
    long long hs[15];
    d2hSync(hs, st.p, sizeof hs);
    double p = 1.0;
    for (int sc = 0; sc < 5; ++sc, p *= 10.0) {
      if (hs[3 * sc] & 0xffffffffll) continue;  // not every value is exact at this scale
      long long mn = hs[3 * sc + 1], mx = hs[3 * sc + 2];
      if (mn > mx) mn = mx = 0;
      const unsigned long long range = (unsigned long long)(mx - mn);
      const int e = range < 0xFFFFull ? 5 : range < 0xFFFFFFFFull ? 6 : 0;
      if (!e) return;
      const int w = e == 5 ? 2 : 4;
      const int64_t total = WS_ENC_HEADER + n * w + 16;
      DBuf<uint8_t> buf(total);
      WS_CK(cudaMemsetAsync(buf.p, 0, total, stream()));
      uint8_t* hdr = pinnedStage(16);
      memcpy(hdr, &mn, 8);
      memcpy(hdr + 8, &p, 8);
      h2dAsync(buf.p, hdr, 16);
      stageCopied();
      WS_LAUNCH(kDecimalEncode, gridFor(n), 256, 0, x, n, p, mn, w, buf.p + WS_ENC_HEADER);
      finish(buf, total, e);
      return;
    }
  });
}

}  // extern "C"
