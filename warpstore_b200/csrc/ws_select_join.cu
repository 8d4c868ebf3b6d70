// Selection (filter -> ascending row indices), gathers and inner hash joins
// (reference: src/gpu.cu:664-800 gpuSelect / gpuSelectMulti / gpuGatherMulti, :1089-1193 gpuHashJoinParts).
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

__global__ void kScanTiles(int64_t* counts, int64_t n) {  // exclusive scan in place, total in counts[n]
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

// per-batch selected counts from the scanned tile offsets: out[b] = offs[tileStart[b+1]] - offs[tileStart[b]]
__global__ void kBatchCounts(const int64_t* offs, const int64_t* tileStart, int nb, int64_t* out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
    out[b] = offs[tileStart[b + 1]] - offs[tileStart[b]];
}

// dst[j] = row idx[j] of the concatenated batches; batch found by binary search of the offsets.
__global__ void kGatherMulti(const ws_col_view* src, const int64_t* boff, int nb, int ptype, int esize,
                             const int32_t* idx, int64_t m, uint8_t* dst) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = idx[j];
    int lo = 0, hi = nb - 1;  // last batch with boff <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(boff + mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    const ws_col_view v = src[lo];
    const int64_t r = g - __ldg(boff + lo);
    if (v.enc) {
      if (ptype == WS_PT_F64) ((double*)dst)[j] = colDblAt(v, r);
      else if (ptype == WS_PT_I32) ((int32_t*)dst)[j] = (int32_t)colIntAt(v, r);
      else ((int64_t*)dst)[j] = colIntAt(v, r);
    } else if (esize == 4) {
      ((int32_t*)dst)[j] = __ldg((const int32_t*)v.p + r);
    } else if (esize == 8) {
      ((int64_t*)dst)[j] = __ldg((const int64_t*)v.p + r);
    } else {
      const uint8_t* s = (const uint8_t*)v.p + r * esize;
      for (int k = 0; k < esize; ++k) dst[j * esize + k] = s[k];
    }
  }
}
__global__ void kGather(const uint8_t* src, int esize, const int32_t* idx, int64_t m, uint8_t* dst) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx[j];
    if (esize == 4) ((int32_t*)dst)[j] = __ldg((const int32_t*)src + r);
    else ((int64_t*)dst)[j] = __ldg((const int64_t*)src + r);
  }
}

// ---------------------------------------------------------------- hash join
// Table: cap (power of two) slots of {int64 key, int32 build row, pad} (16 bytes, one sector per
// probe step); empty = INT64_MIN (the BIGINT NULL sentinel, never inserted).  Linear probing from
// mix64(key).  Keys: I32 views widen to int64 (their sentinel is NULL), I64 views as stored, F64 views
// (bit patterns converted by the engine) truncated, NaN = NULL (src/gpu.cu:180-202).
constexpr long long kJEmpty = (long long)0x8000000000000000ull;
struct JSlot {
  long long key;
  int row;
  int pad;
};

__device__ __forceinline__ bool joinKey(const ws_col_view& c, int64_t r, long long& k) {
  if (c.t == 0 || c.t == 3) {
    const int v = __ldg((const int*)c.p + r);
    k = v;
    return v != WS_NULL_I32;
  }
  if (c.t == 1 || c.t == 4) {
    k = __ldg((const long long*)c.p + r);
    return k != WS_NULL_I64;
  }
  const double d = __ldg((const double*)c.p + r);
  k = (long long)d;
  return d == d;
}

__global__ void kJoinInit(JSlot* t, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    t[i].key = kJEmpty, t[i].row = -1;
}

// Inserts build rows [base, base + n); `bounded` probe steps at most (the table has >= 2n slots, so
// an insert meets an empty slot within cap steps; err is raised otherwise).
__global__ void kJoinBuild(ws_col_view key, int64_t base, int64_t n, JSlot* t, u64 mask, int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    long long k;
    if (!joinKey(key, base + i, k)) continue;
    u64 s = mix64((u64)k) & mask;
    bool done = false;
    for (u64 p = 0; p <= mask; ++p) {
      const long long prev = (long long)atomicCAS((u64*)&t[s].key, (u64)kJEmpty, (u64)k);
      if (prev == kJEmpty) {
        t[s].row = (int)(base + i);
        done = true;
        break;
      }
      s = (s + 1) & mask;
    }
    if (!done) *err = 1;
  }
}

// Probe rows [base, base + n): every match becomes a pair.  Lanes keep up to kKeep matches in
// registers; a warp reserves its output with one atomic on the partition's counter (pairs of a warp
// are contiguous).  With count != null (exact sizing pass) only the matches are counted.
constexpr int kKeep = 4;
__global__ void kJoinProbe(ws_col_view key, int64_t base, int64_t n, const JSlot* t, u64 mask, int64_t outBase,
                           int64_t capacity, unsigned long long* counter, int32_t* ob, int32_t* op) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    int c = 0;
    int keep[kKeep];
    long long k = 0;
    u64 s0 = 0;
    bool valid = i < n && joinKey(key, base + i, k);
    if (valid) {
      s0 = mix64((u64)k) & mask;
      u64 s = s0;
      for (u64 p = 0; p <= mask; ++p) {
        const JSlot e = t[s];
        if (e.key == kJEmpty) break;
        if (e.key == k) {
          if (c < kKeep) keep[c] = e.row;
          ++c;
        }
        s = (s + 1) & mask;
      }
    }
    // warp exclusive prefix of c, one reservation per warp
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long wbase = 0;
    if (lane == 0 && total) wbase = atomicAdd(counter, (unsigned long long)total);
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    if (!ob || c == 0) continue;
    int64_t o = (int64_t)wbase + incl - c;
    if (o + c > capacity) continue;  // sized too small: the host reruns with the exact count
    const int32_t pr = (int32_t)(base + i);
    if (c <= kKeep) {
      for (int j = 0; j < c; ++j) ob[outBase + o + j] = keep[j], op[outBase + o + j] = pr;
    } else {
      u64 s = s0;
      for (u64 p = 0; p <= mask; ++p) {
        const JSlot e = t[s];
        if (e.key == kJEmpty) break;
        if (e.key == k) ob[outBase + o] = e.row, op[outBase + o] = pr, ++o;
        s = (s + 1) & mask;
      }
    }
  }
}

}  // namespace

// Batch descriptor upload shared with the aggregator (ws_ops.cu).
struct SelDesc {
  DBuf<uint8_t> buf;
  int64_t ntiles = 0;
  const ws_col_view* cols;
  const int64_t *n, *tileStart, *rowStart;
  const uint32_t* const* del;
  const TProgs* progs;
};

static SelDesc uploadSel(int nb, int ncols, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                         const TProgs* progs) {
  SelDesc d;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = (off + 15) & ~(size_t)15;
    off = o + bytes;
    return o;
  };
  const size_t oCols = take((size_t)nb * ncols * sizeof(ws_col_view)), oN = take(8 * nb), oDel = take(8 * nb),
               oTile = take(8 * (nb + 1)), oRow = take(8 * (nb + 1)), oProg = progs ? take(sizeof(TProgs)) : 0;
  uint8_t* st = pinnedStage(off);
  memcpy(st + oCols, bcols, (size_t)nb * ncols * sizeof(ws_col_view));
  int64_t* n = (int64_t*)(st + oN);
  const uint32_t** del = (const uint32_t**)(st + oDel);
  int64_t *ts = (int64_t*)(st + oTile), *rs = (int64_t*)(st + oRow);
  ts[0] = rs[0] = 0;
  for (int b = 0; b < nb; ++b) {
    n[b] = bn[b];
    del[b] = bdel ? bdel[b] : nullptr;
    ts[b + 1] = ts[b] + (bn[b] + kTile - 1) / kTile;
    rs[b + 1] = rs[b] + bn[b];
  }
  d.ntiles = ts[nb];
  if (progs) memcpy(st + oProg, progs, sizeof(TProgs));
  d.buf = DBuf<uint8_t>((int64_t)off);
  h2dAsync(d.buf.p, st, off);
  stageCopied();
  uint8_t* p = d.buf.p;
  d.cols = (const ws_col_view*)(p + oCols);
  d.n = (const int64_t*)(p + oN);
  d.del = (const uint32_t* const*)(p + oDel);
  d.tileStart = (const int64_t*)(p + oTile);
  d.rowStart = (const int64_t*)(p + oRow);
  d.progs = progs ? (const TProgs*)(p + oProg) : nullptr;
  return d;
}

// Runs the two selection passes; returns the selected count, writes per-batch counts (host) and the
// indices (device, into *out or a new buffer when *out is null).
static int64_t selectRun(const ws_expr_env& env, bool hasWhere, ws_prog where, int nb, const int64_t* bn,
                         const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int32_t** out,
                         int64_t* perBatch, const ws_jit_program* jit) {
  for (int b = 0; b < nb; ++b)
    if (perBatch) perBatch[b] = 0;
  int64_t total = 0;
  for (int b = 0; b < nb; ++b) total += bn[b];
  if (total <= 0) return 0;
  ws_agg_plan fp;
  memset(&fp, 0, sizeof fp);
  fp.hasWhere = hasWhere;
  fp.where = where;
  fp.naggs = 1;
  fp.ops[0] = WS_AGG_COUNT;
  const bool useJit = jit && jit->state.load() == 1 && jit->kernels.fn[K_SELECT_COUNT] && [&] {
    for (int b = 0; b < nb; ++b)
      for (int c = 0; c < ncols; ++c)
        if (bcols[(int64_t)b * ncols + c].enc && !env.cols[c].enc) return false;
    return true;
  }();
  std::unique_ptr<TProgs> progs;
  if (!useJit) {
    progs.reset(new TProgs);
    buildTProgs(env, ncols, fp, hasWhere, *progs);
  }
  SelDesc d = uploadSel(nb, ncols, bn, bdel, bcols, progs.get());
  Launch L;
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
  L.naggs = 1;
  L.rowWords = 1;
  const KernelSet& ks = useJit ? jit->kernels : interpKernels();
  DBuf<int64_t> counts(d.ntiles + 1);
  L.tileCount = (i64*)counts.p;
  launchScan(ks.fn[K_SELECT_COUNT], persistentGrid(ks.fn[K_SELECT_COUNT], 0, d.ntiles), 0, L);
  WS_LAUNCH(kScanTiles, 1, 1024, 0, counts.p, d.ntiles);
  DBuf<int64_t> pb(nb);
  WS_LAUNCH(kBatchCounts, gridFor(nb), 256, 0, counts.p, d.tileStart, nb, pb.p);
  int64_t m = 0;
  WS_CK(cudaMemcpyAsync(&m, counts.p + d.ntiles, 8, cudaMemcpyDeviceToHost, stream()));
  std::vector<int64_t> per(nb);
  WS_CK(cudaMemcpyAsync(per.data(), pb.p, 8 * nb, cudaMemcpyDeviceToHost, stream()));
  sync();
  if (perBatch) memcpy(perBatch, per.data(), 8 * nb);
  if (m > INT32_MAX) throw Error("selection too large (>2^31 rows)", WS_ERR_INTERNAL);
  if (!*out) *out = (int32_t*)tmpAlloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (m) {
    L.outIdx = *out;
    launchScan(ks.fn[K_SELECT_WRITE], persistentGrid(ks.fn[K_SELECT_WRITE], 0, d.ntiles), 0, L);
  }
  return m;
}

}  // namespace ws

using namespace ws;

extern "C" {

int ws_select(const ws_expr_env* env, int has_where, ws_prog where, int64_t n, const uint32_t* del, int32_t* out_idx,
              const ws_jit_program* jit, int64_t* count) {
  return guardedCall([&] {
    const uint32_t* dels[1] = {del};
    int32_t* o = out_idx;
    if (n <= 0) {
      *count = 0;
      return;
    }
    if (!out_idx) throw Error("ws_select needs an output buffer of n indices", WS_ERR_ARG);
    *count = selectRun(*env, has_where != 0, where, 1, &n, dels, env->cols, WS_MAX_COLS, &o, nullptr, jit);
  });
}

int ws_select_multi(const ws_expr_env* env, int has_where, ws_prog where, int nb, const int64_t* bn,
                    const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int32_t** out_idx,
                    int64_t* per_batch, const ws_jit_program* jit, int64_t* count) {
  return guardedCall([&] {
    *out_idx = nullptr;
    int32_t* o = nullptr;
    *count = selectRun(*env, has_where != 0, where, nb, bn, bdel, bcols, ncols, &o, per_batch, jit);
    if (!o) o = (int32_t*)tmpAlloc(4);
    *out_idx = o;
  });
}

int ws_gather_multi(const ws_col_view* src, const int64_t* boff, int nb, int ptype, int esize, const int32_t* idx,
                    int64_t m, void* dst) {
  return guardedCall([&] {
    if (m <= 0) return;
    std::vector<ws_col_view> vs(src, src + nb);
    for (auto& v : vs) v.t = ptype == WS_PT_I32 ? 3 : ptype == WS_PT_I64 ? 4 : 2;  // encoded: NULL sentinels as stored
    const size_t vb = (size_t)nb * sizeof(ws_col_view), bytes = vb + 8 * (size_t)nb;
    uint8_t* st = pinnedStage(bytes);
    memcpy(st, vs.data(), vb);
    memcpy(st + vb, boff, 8 * (size_t)nb);
    DBuf<uint8_t> d((int64_t)bytes);
    h2dAsync(d.p, st, bytes);
    stageCopied();
    WS_LAUNCH(kGatherMulti, (unsigned)std::min<int64_t>((m + 255) / 256, (int64_t)smCount() * 16), 256, 0,
              (const ws_col_view*)d.p, (const int64_t*)(d.p + vb), nb, ptype, esize, idx, m, (uint8_t*)dst);
  });
}

int ws_gather(const void* src, int ptype, const int32_t* idx, int64_t m, void* dst) {
  return guardedCall([&] {
    if (m <= 0) return;
    WS_LAUNCH(kGather, gridFor(m), 256, 0, (const uint8_t*)src, ptype == WS_PT_I32 ? 4 : 8, idx, m, (uint8_t*)dst);
  });
}

int ws_hash_join_parts(ws_col_view build_key, const int64_t* boff, int nbparts, ws_col_view probe_key,
                       const int64_t* poff, int npparts, int32_t** out_build, int32_t** out_probe, int64_t* out_off,
                       int64_t* m_out) {
  return guardedCall([&] {
    *out_build = *out_probe = nullptr;
    const int pb = nbparts, pp = npparts;
    if (pb < 1 || pp < 1 || (pb != 1 && pb != pp)) throw Error("internal: partition count mismatch in join", WS_ERR_INTERNAL);
    const int64_t nb = boff[pb], np = poff[pp];
    if (out_off)
      for (int p = 0; p <= pp; ++p) out_off[p] = 0;
    *m_out = 0;
    if (nb == 0 || np == 0) {
      *out_build = (int32_t*)tmpAlloc(4);
      *out_probe = (int32_t*)tmpAlloc(4);
      return;
    }
    std::vector<int64_t> reg(pb + 1, 0), cap(pb);
    for (int q = 0; q < pb; ++q) {
      int64_t c = 2;
      while (c < (boff[q + 1] - boff[q]) * 2) c <<= 1;
      cap[q] = c;
      reg[q + 1] = reg[q] + c;
    }
    DBuf<JSlot> table(reg[pb]);
    DBuf<int> err(1);
    WS_CK(cudaMemsetAsync(err.p, 0, 4, stream()));
    WS_LAUNCH(kJoinInit, gridFor(reg[pb]), 256, 0, table.p, reg[pb]);
    for (int q = 0; q < pb; ++q) {
      const int64_t n = boff[q + 1] - boff[q];
      if (n) WS_LAUNCH(kJoinBuild, gridFor(n), 256, 0, build_key, boff[q], n, table.p + reg[q], (u64)(cap[q] - 1), err.p);
    }
    // One probe pass with output capacity = probe rows per partition (enough for every join whose
    // build keys are unique); if a partition produced more, a second pass writes with exact sizes.
    std::vector<int64_t> capOut(pp), outStart(pp + 1, 0);
    for (int p = 0; p < pp; ++p) {
      capOut[p] = poff[p + 1] - poff[p];
      outStart[p + 1] = outStart[p] + capOut[p];
    }
    DBuf<unsigned long long> counters(pp);
    std::vector<unsigned long long> cnt(pp);
    for (int pass = 0; pass < 2; ++pass) {
      WS_CK(cudaMemsetAsync(counters.p, 0, 8 * pp, stream()));
      DBuf<int32_t> ob(std::max<int64_t>(outStart[pp], 1)), op(std::max<int64_t>(outStart[pp], 1));
      for (int p = 0; p < pp; ++p) {
        const int q = pb == 1 ? 0 : p;
        const int64_t n = poff[p + 1] - poff[p];
        if (n)
          WS_LAUNCH(kJoinProbe, gridFor(n), 256, 0, probe_key, poff[p], n, table.p + reg[q], (u64)(cap[q] - 1),
                    outStart[p], capOut[p], counters.p + p, ob.p, op.p);
      }
      int e = 0;
      WS_CK(cudaMemcpyAsync(cnt.data(), counters.p, 8 * pp, cudaMemcpyDeviceToHost, stream()));
      WS_CK(cudaMemcpyAsync(&e, err.p, 4, cudaMemcpyDeviceToHost, stream()));
      sync();
      if (e) throw Error("internal: join hash table full", WS_ERR_INTERNAL);
      bool fits = true;
      int64_t m = 0;
      for (int p = 0; p < pp; ++p) {
        fits &= (int64_t)cnt[p] <= capOut[p];
        m += (int64_t)cnt[p];
      }
      if (m > INT32_MAX) throw Error("join result too large (>2^31 rows)", WS_ERR_INTERNAL);
      if (fits) {
        // make the partitions' pairs contiguous
        std::vector<int64_t> dst(pp + 1, 0);
        for (int p = 0; p < pp; ++p) dst[p + 1] = dst[p] + (int64_t)cnt[p];
        if (pp == 1 || dst == outStart) {
          *out_build = ob.release();
          *out_probe = op.release();
        } else {
          DBuf<int32_t> cb(std::max<int64_t>(m, 1)), cp(std::max<int64_t>(m, 1));
          for (int p = 0; p < pp; ++p)
            if (cnt[p]) {
              WS_CK(cudaMemcpyAsync(cb.p + dst[p], ob.p + outStart[p], 4 * cnt[p], cudaMemcpyDeviceToDevice, stream()));
              WS_CK(cudaMemcpyAsync(cp.p + dst[p], op.p + outStart[p], 4 * cnt[p], cudaMemcpyDeviceToDevice, stream()));
            }
          *out_build = cb.release();
          *out_probe = cp.release();
        }
        if (out_off)
          for (int p = 0; p <= pp; ++p) out_off[p] = dst[p];
        *m_out = m;
        return;
      }
      for (int p = 0; p < pp; ++p) {  // exact sizes for the second pass
        capOut[p] = (int64_t)cnt[p];
        outStart[p + 1] = outStart[p] + capOut[p];
      }
    }
    throw Error("internal: join output sizing failed", WS_ERR_INTERNAL);
  });
}

int ws_hash_join(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int32_t** out_build,
                 int32_t** out_probe, int64_t* m) {
  const int64_t bo[2] = {0, nb}, po[2] = {0, np};
  return ws_hash_join_parts(build_key, bo, 1, probe_key, po, 1, out_build, out_probe, nullptr, m);
}

}  // extern "C"
