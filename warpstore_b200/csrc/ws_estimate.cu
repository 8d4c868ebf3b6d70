// Cardinality estimation for sizing hash tables: a HyperLogLog sketch of a strided sample of the
// filtered GROUP BY keys (one pass over the sampled rows, registers combined by shared then global
// atomic max), and the inference of a small MLP (BF16 weights, FP32 accumulation) that maps sketch and
// table statistics to the predicted group count.  No counterpart in the reference, which sizes tables
// from dictionary sizes and segment min/max alone (src/engine_select.cpp:1154-1167).
#include <cuda_bf16.h>

#include <cstring>

#include "ws_internal.h"
#include "ws_interp.cuh"

namespace ws {
namespace {

constexpr int kHllMaxP = 12;  // 4096 registers (16 KB of shared memory)

struct SketchSpec {
  const TInstr* code;
  int where[2];            // start, len (len 0: no filter)
  int keys[WS_MAX_KEYS][2];
  int keyInt[WS_MAX_KEYS];
  int whereInt;            // the filter's result type (1: integer boolean, 0: 3-valued double)
  int nkeys, ncols, nb, p;
  const ws_col_view* cols;  // [nb][ncols]
  const int64_t* rowStart;  // [nb + 1]
  const uint32_t* const* del;
  int64_t samples;          // sampled global rows: k * stride, k < samples
  int64_t stride;
};

// The HLL hash of a row's key word(s): one key -> mix64 of its bits (int64 value or canonical double
// bits); several keys -> the GROUP BY hash fold (the key word of multi-key groups), mixed once more.
__device__ __forceinline__ u64 sketchHash(const SketchSpec& s, const ws_col_view* cv, i64 r, const EnvK& env) {
  u64 h = 0x9e3779b97f4a7c15ull;
  u64 one = 0;
  for (int k = 0; k < s.nkeys; ++k) {
    const Word w = vmRun(s.code, s.keys[k][0], s.keys[k][1], cv, r, env);
    const u64 b = s.keyInt[k] ? (u64)w.i : (u64)dkeyBits(w.d);
    one = b;
    h = mix64(h ^ b) + (u64)k;
  }
  return mix64(s.nkeys == 1 ? one : h);
}

// regs[j] = max rank of the sampled hashes with top-p bits j; counts = {sampled rows, passing rows}
__global__ void kHllSketch(const __grid_constant__ SketchSpec s, const __grid_constant__ EnvK env, unsigned* regs,
                           unsigned long long* counts) {
  __shared__ unsigned sr[1 << kHllMaxP];
  const int m = 1 << s.p;
  for (int j = threadIdx.x; j < m; j += blockDim.x) sr[j] = 0;
  __syncthreads();
  unsigned long long sampled = 0, passing = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < s.samples; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = k * s.stride;
    int lo = 0, hi = s.nb - 1;  // batch of global row g: last with rowStart <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(s.rowStart + mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    const i64 r = g - __ldg(s.rowStart + lo);
    const uint32_t* del = s.del[lo];
    if (del && ((__ldg(del + (r >> 5)) >> (r & 31)) & 1u)) continue;
    ++sampled;
    const ws_col_view* cv = s.cols + (int64_t)lo * s.ncols;
    if (s.where[1]) {
      const Word w = vmRun(s.code, s.where[0], s.where[1], cv, r, env);
      if (!(s.whereInt ? w.i != 0 : truthy(w.d))) continue;
    }
    ++passing;
    if (!s.nkeys) continue;  // counting only: the filter's sampled selectivity
    const u64 h = sketchHash(s, cv, r, env);
    const unsigned j = (unsigned)(h >> (64 - s.p));
    const u64 rest = h << s.p;
    const unsigned rank = rest ? (unsigned)__clzll(rest) + 1u : (unsigned)(64 - s.p + 1);
    atomicMax(&sr[j], rank);
  }
  for (int o = 16; o; o >>= 1) {
    sampled += __shfl_xor_sync(0xffffffffu, sampled, o);
    passing += __shfl_xor_sync(0xffffffffu, passing, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counts, sampled);
    atomicAdd(counts + 1, passing);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < m; j += blockDim.x)
    if (sr[j]) atomicMax(regs + j, sr[j]);
}

// One block per input row of features: h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), y = h2 W3 + b3.
// W1 [F][H], W2 [H][H], W3 [H] in BF16; biases and accumulation in FP32.  H = blockDim.x <= 128.
__global__ void kMlp(const float* x, int F, int H, const __nv_bfloat16* W1, const float* b1, const __nv_bfloat16* W2,
                     const float* b2, const __nv_bfloat16* W3, float b3, float* y) {
  __shared__ float xs[64], h1[128], part[4];
  const int j = threadIdx.x, q = blockIdx.x;
  for (int i = j; i < F; i += blockDim.x) xs[i] = x[(int64_t)q * F + i];
  __syncthreads();
  float a = b1[j];
  for (int i = 0; i < F; ++i) a = fmaf(xs[i], __bfloat162float(W1[i * H + j]), a);
  h1[j] = fmaxf(a, 0.f);
  __syncthreads();
  float c = b2[j];
  for (int i = 0; i < H; ++i) c = fmaf(h1[i], __bfloat162float(W2[i * H + j]), c);
  float v = fmaxf(c, 0.f) * __bfloat162float(W3[j]);
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((j & 31) == 0) part[j >> 5] = v;
  __syncthreads();
  if (j == 0) {
    float t = b3;
    for (int w = 0; w < (H + 31) / 32; ++w) t += part[w];
    y[q] = t;
  }
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

int ws_hll_sketch(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int nb, const int64_t* bn,
                  const uint32_t* const* bdel, const ws_col_view* bcols, int p, int64_t sample_rows, uint32_t* regs_out,
                  int64_t* sampled, int64_t* passing) {
  return guardedCall([&] {
    if (ncols < 0 || ncols > WS_MAX_COLS || nb < 0) throw Error("sketch: bad column or batch count", WS_ERR_ARG);
    if (p < 4 || p > kHllMaxP) throw Error("sketch: precision must be 4..12", WS_ERR_ARG);
    if (plan->nkeys < 0 || plan->nkeys > WS_INTERP_KEYS) throw Error("sketch: 0 to 4 GROUP BY keys", WS_ERR_ARG);
    std::unique_ptr<TProgs> tp(new TProgs);
    buildTProgs(*env, ncols, *plan, plan->hasWhere != 0, *tp);
    SketchSpec s{};
    memcpy(s.where, tp->where, sizeof s.where);
    memcpy(s.keys, tp->keys, sizeof s.keys);
    for (int k = 0; k < plan->nkeys; ++k) s.keyInt[k] = typeProg(*env, plan->keys[k], ncols).isInt() ? 1 : 0;
    s.whereInt = plan->hasWhere ? (typeProg(*env, plan->where, ncols).isInt() ? 1 : 0) : 1;
    s.nkeys = plan->nkeys;
    s.ncols = ncols;
    s.nb = nb;
    s.p = p;
    std::vector<int64_t> rs(nb + 1, 0);
    for (int b = 0; b < nb; ++b) rs[b + 1] = rs[b] + bn[b];
    const int64_t total = rs[nb];
    s.stride = std::max<int64_t>(1, sample_rows > 0 ? total / std::max<int64_t>(sample_rows, 1) : 1);
    s.samples = total ? (total + s.stride - 1) / s.stride : 0;
    // device copies: programs, views, row starts, bitmaps
    const size_t codeBytes = sizeof(TInstr) * 1024, colBytes = sizeof(ws_col_view) * (size_t)nb * ncols,
                 rsBytes = 8 * (size_t)(nb + 1), delBytes = sizeof(void*) * (size_t)nb;
    const size_t total_b = codeBytes + colBytes + rsBytes + delBytes + 64;
    DBuf<uint8_t> dbuf((int64_t)total_b);
    uint8_t* st = pinnedStage(total_b);
    size_t off = 0;
    memcpy(st + off, tp->code, codeBytes);
    s.code = (const TInstr*)(dbuf.p + off);
    off += codeBytes;
    memcpy(st + off, bcols, colBytes);
    s.cols = (const ws_col_view*)(dbuf.p + off);
    off += (colBytes + 15) & ~(size_t)15;
    memcpy(st + off, rs.data(), rsBytes);
    s.rowStart = (const int64_t*)(dbuf.p + off);
    off += (rsBytes + 15) & ~(size_t)15;
    for (int b = 0; b < nb; ++b) ((const uint32_t**)(st + off))[b] = bdel ? bdel[b] : nullptr;
    s.del = (const uint32_t* const*)(dbuf.p + off);
    off += delBytes;
    h2dAsync(dbuf.p, st, off);
    stageCopied();
    DBuf<unsigned> regs(1 << p);
    DBuf<unsigned long long> counts(2);
    WS_CK(cudaMemsetAsync(regs.p, 0, 4u << p, stream()));
    WS_CK(cudaMemsetAsync(counts.p, 0, 16, stream()));
    if (s.samples) {
      const int64_t g = std::min<int64_t>((s.samples + 255) / 256, (int64_t)smCount() * 4);
      kHllSketch<<<(unsigned)std::max<int64_t>(g, 1), 256, 0, stream()>>>(s, envK(*env), regs.p, counts.p);
      WS_CK(cudaGetLastError());
      countLaunch();
    }
    unsigned long long hc[2];
    WS_CK(cudaMemcpyAsync(regs_out, regs.p, 4u << p, cudaMemcpyDeviceToHost, stream()));
    WS_CK(cudaMemcpyAsync(hc, counts.p, 16, cudaMemcpyDeviceToHost, stream()));
    sync();
    *sampled = (int64_t)hc[0];
    *passing = (int64_t)hc[1];
  });
}

int ws_mlp_infer(const float* x, int rows, int features, int hidden, const uint16_t* w1_bf16, const float* b1,
                 const uint16_t* w2_bf16, const float* b2, const uint16_t* w3_bf16, float b3, float* y) {
  return guardedCall([&] {
    if (features < 1 || features > 64 || hidden < 32 || hidden > 128 || hidden % 32)
      throw Error("mlp: 1..64 features, 32..128 hidden units (a multiple of 32)", WS_ERR_ARG);
    if (rows <= 0) return;
    const size_t xb = 4 * (size_t)rows * features, w1b = 2 * (size_t)features * hidden, b1b = 4 * (size_t)hidden,
                 w2b = 2 * (size_t)hidden * hidden, b2b = 4 * (size_t)hidden, w3b = 2 * (size_t)hidden;
    const size_t tot = xb + w1b + b1b + w2b + b2b + w3b + 96;
    DBuf<uint8_t> d((int64_t)tot);
    DBuf<float> dy(rows);
    uint8_t* st = pinnedStage(tot);
    size_t off = 0;
    auto put = [&](const void* src, size_t n) {
      memcpy(st + off, src, n);
      const size_t at = off;
      off += (n + 15) & ~(size_t)15;
      return d.p + at;
    };
    const float* dx = (const float*)put(x, xb);
    const __nv_bfloat16* dw1 = (const __nv_bfloat16*)put(w1_bf16, w1b);
    const float* db1 = (const float*)put(b1, b1b);
    const __nv_bfloat16* dw2 = (const __nv_bfloat16*)put(w2_bf16, w2b);
    const float* db2 = (const float*)put(b2, b2b);
    const __nv_bfloat16* dw3 = (const __nv_bfloat16*)put(w3_bf16, w3b);
    h2dAsync(d.p, st, off);
    stageCopied();
    kMlp<<<rows, hidden, 0, stream()>>>(dx, features, hidden, dw1, db1, dw2, db2, dw3, b3, dy.p);
    WS_CK(cudaGetLastError());
    countLaunch();
    d2hSync(y, dy.p, 4 * (size_t)rows);
  });
}

}  // extern "C"
