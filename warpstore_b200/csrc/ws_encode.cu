// Segment encoding on the GPU (the flush path of the engine's storage: src/storage.cu:1138-1192 encodes
// segment columns on the host): integer columns to the bit-packed (enc 7) or run-length (enc 8)
// formats that the scan kernels decode (formats: ws_dev.cuh).
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

}  // extern "C"
