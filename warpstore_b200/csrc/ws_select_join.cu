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
// Keys are hashed with h = mix64(key).  The stored key is key ^ 2^63, so an all-zero slot is empty:
// the one key that maps to 0 is INT64_MIN, the BIGINT NULL sentinel, which is never inserted.  The
// table's layout (buckets of keys, rows apart) is described at jBucket below.
//
// A build side whose table would not stay in L2 is split into P = 2^b passes by the top b bits of h:
// pass p builds the table of the build keys with h >> (64 - b) == p (reusing one buffer) and probes
// every probe row, skipping the rows of the other passes.  Each pass's random table accesses then hit
// L2; the probe keys are re-read P times as a sequential stream (loaded with the evict-first hint so
// that they do not push the table out).
// Keys: I32 views widen to int64 (their sentinel is NULL), I64 views as stored, F64 views (bit
// patterns converted by the engine) truncated, NaN = NULL (src/gpu.cu:180-202).
constexpr u64 kJSign = 0x8000000000000000ull;

__device__ __forceinline__ bool joinKeyStream(const ws_col_view& c, int64_t r, long long& k) {
  if (c.t == 0 || c.t == 3) {
    const int v = __ldcs((const int*)c.p + r);
    k = v;
    return v != WS_NULL_I32;
  }
  if (c.t == 1 || c.t == 4) {
    k = __ldcs((const long long*)c.p + r);
    return k != WS_NULL_I64;
  }
  const double d = __ldcs((const double*)c.p + r);
  k = (long long)d;
  return d == d;
}

// Hash table: buckets of 64 bytes, each 4 keys in its first 32-byte sector (key ^ 2^63; 0 = empty) and
// their 4 build rows (int32) in the second, read only when a slot matched.  A random DRAM access brings
// 64 bytes whatever is asked for, so the rows beside the keys arrive with them: a match's row is an L2
// hit instead of a second random DRAM access (rows in a separate array cost ~117 DRAM bytes per probe).
// The bucket of a key is the low 32 bits of its hash scaled to the bucket count (any count: the table
// is sized to the keys, not to a power of two); a full bucket overflows into the next one, so a probe
// walks buckets from the key's own until one has an empty slot.  A probe costs one 256-bit load when
// its bucket is not full.
constexpr u64 kJBucketWords = 8;  // u64 words per bucket: keys [0, 4), rows as int32 in [4, 6)
constexpr u64 kJRowStride = 16;   // int32 per bucket, for the rows' view of the table (starting at word 4)
__device__ __forceinline__ u64 jBucket(u64 h, u64 nbuckets) {
  return nbuckets <= 0xffffffffull ? (u64)__umulhi((unsigned)h, (unsigned)nbuckets)
                                   : ((h & 0xffffffffull) * nbuckets) >> 32;
}
// L2 policy for the bucket loads: keep the key table resident while the probe keys stream past
__device__ __forceinline__ u64 jKeepPolicy() {
  u64 pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void ldBucket(const u64* p, u64 pol, u64 (&k)[4]) {
  asm("ld.global.nc.L2::cache_hint.v4.u64 {%0,%1,%2,%3}, [%4], %5;"
      : "=l"(k[0]), "=l"(k[1]), "=l"(k[2]), "=l"(k[3])
      : "l"(p), "l"(pol));
}

// Key filter of an inner join's build side (a blocked Bloom filter that L2 holds: 16 bits per build key
// in 64-bit words): a key sets 4 bits of one word, chosen by other bits of its hash than its bucket's;
// a probe key whose 4 bits are not all set has no match and skips its bucket's random DRAM access.
struct JFilter {
  u64* words;  // null: no filter
  u64 mask;    // words - 1 (a power of two)
};
__device__ __forceinline__ u64 jFilterBits(u64 h) {
  return (1ull << (h & 63)) | (1ull << ((h >> 6) & 63)) | (1ull << ((h >> 12) & 63)) | (1ull << ((h >> 18) & 63));
}
__device__ __forceinline__ u64 jFilterWord(u64 h, u64 mask) { return (h >> 32) & mask; }
__device__ __forceinline__ u64 ldFilter(const u64* p, u64 pol) {
  u64 v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
  return v;
}

struct JPass {
  int bits;  // log2 of the pass count
  int pass;
  __device__ __forceinline__ bool mine(u64 h) const { return bits == 0 || (int)(h >> (64 - bits)) == pass; }
};

// Build-key statistics of one build partition: st[0] = non-NULL keys, st[1] = min, st[2] = max (as
// int64), st[3 + p] = keys of hash pass p (when bits > 0).  kJoinStatsInit sets the identities.
constexpr int kJStatWords = 3 + 64;
__global__ void kJoinStatsInit(unsigned long long* st) {
  const int i = threadIdx.x;
  if (i < kJStatWords) st[i] = i == 1 ? 0x7fffffffffffffffull : i == 2 ? 0x8000000000000000ull : 0ull;
}

__global__ void kJoinStats(ws_col_view key, int64_t base, int64_t n, int bits, unsigned long long* st) {
  __shared__ unsigned long long h[64];
  __shared__ unsigned long long cnt;
  __shared__ long long mn, mx;
  const int P = 1 << bits;
  for (int i = threadIdx.x; i < P; i += blockDim.x) h[i] = 0;
  if (threadIdx.x == 0) cnt = 0, mn = 0x7fffffffffffffffll, mx = (long long)0x8000000000000000ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  long long lmn = 0x7fffffffffffffffll, lmx = (long long)0x8000000000000000ull;
  unsigned long long lc = 0;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    long long k = 0;
    const bool ok = i < n && joinKeyStream(key, base + i, k);
    if (ok) lmn = min(lmn, k), lmx = max(lmx, k), ++lc;
    if (bits) {
      const int part = ok ? (int)(mix64((u64)k) >> (64 - bits)) : -1;
      const unsigned same = __match_any_sync(0xffffffffu, part);
      if (part >= 0 && lane == __ffs(same) - 1) atomicAdd(&h[part], (unsigned long long)__popc(same));
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    lmn = min(lmn, __shfl_xor_sync(0xffffffffu, lmn, o));
    lmx = max(lmx, __shfl_xor_sync(0xffffffffu, lmx, o));
    lc += __shfl_xor_sync(0xffffffffu, lc, o);
  }
  if (lane == 0 && lc) {
    atomicMin(&mn, lmn);
    atomicMax(&mx, lmx);
    atomicAdd(&cnt, lc);
  }
  __syncthreads();
  if (threadIdx.x == 0 && cnt) {
    atomicAdd(&st[0], cnt);
    atomicMin((long long*)&st[1], mn);
    atomicMax((long long*)&st[2], mx);
  }
  for (int i = threadIdx.x; i < P && bits; i += blockDim.x)
    if (h[i]) atomicAdd(&st[3 + i], h[i]);
}

// Coordinated key sample of a join side: the hash mix64(key) of every non-NULL key whose hash is below
// tau, appended (in no order) to out[0, cap); *count receives every qualifying key, also those past cap.
// Both sides sampled with one tau keep exactly the keys of both whose hash is below it, so the join of
// the two samples holds every pair of those keys: a scaled estimate of the join's pairs.
__global__ void kJoinKeySample(ws_col_view key, int64_t n, u64 tau, u64* out, int64_t cap, unsigned long long* count) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    long long k = 0;
    const bool valid = i < n && joinKeyStream(key, i, k);
    const u64 h = mix64((u64)k);
    const bool take = valid && h < tau;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    const int64_t at = (int64_t)base + __popc(m & ((1u << lane) - 1u));
    if (take && at < cap) out[at] = h;
  }
}

// Inserts the pass's build rows of [base, base + n): CAS into the first empty slot of the key's bucket
// or of the buckets after it.  The table has more slots than the pass's keys, so an insert meets an
// empty slot within nbuckets steps; err is raised otherwise.  (Measured: giving each thread several
// rows whose loads overlap ran slower, 0.58 against 0.47 ms for 7.5M keys: the inserts are bound by
// the table's random DRAM traffic, not by their latency.)
__global__ void kJoinBuild(ws_col_view key, int64_t base, int64_t n, JPass jp, u64* keys, int* rows, u64 nbuckets,
                           int* err, JFilter jf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    long long k;
    if (!joinKeyStream(key, base + i, k)) continue;
    const u64 h = mix64((u64)k);
    if (!jp.mine(h)) continue;
    if (jf.words) atomicOr((unsigned long long*)(jf.words + jFilterWord(h, jf.mask)), jFilterBits(h));
    const u64 sk = (u64)k ^ kJSign;
    u64 b = jBucket(h, nbuckets);
    bool done = false;
    for (u64 step = 0; step < nbuckets && !done; ++step) {
      u64* bk = keys + b * kJBucketWords;
      // the bucket through L2 (other threads' inserts are visible there); a slot seen empty may have been
      // taken since: the CAS decides, and a lost CAS moves on to the next slot
      const ulonglong2 lo = __ldcg((const ulonglong2*)bk), hi = __ldcg((const ulonglong2*)bk + 1);
      const u64 seen[4] = {lo.x, lo.y, hi.x, hi.y};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (done || seen[q] != 0ull) continue;
        if (atomicCAS((unsigned long long*)(bk + q), 0ull, sk) == 0ull) {
          rows[b * kJRowStride + q] = (int)(base + i);
          done = true;
        }
      }
      b = b + 1 == nbuckets ? 0 : b + 1;
    }
    if (!done) *err = 1;
  }
}

// ---- output: pairs staged per warp in shared memory, flushed with one atomic on the partition's
// counter per flush (coalesced writes).  Pairs at or past `capacity` are not written: the host
// reruns with the exact count.
constexpr int kJThreads = 256, kJPer = 4, kJStage = 256;
constexpr int kJHashPer = 2;  // probe rows per lane and step of the hash probe (1 and 4 measured slower)
constexpr int kJWarps = kJThreads / 32;

struct JOut {
  int32_t* ob;
  int32_t* op;
  int64_t outBase, capacity;
  unsigned long long* counter;
  int outer;         // every probe row without a match gives one pair (-1, probe row)
  uint8_t* matched;  // non-null: matched[build row - rowBase] = 1 for every build row that matched
  int64_t rowBase;   // first build row of the partition (matched[] index base)
};

// Writes the warp's staged pairs [0, fill) (all lanes of the warp call it).
__device__ __forceinline__ void jFlush(const JOut& o, const int2* st, int fill, int lane) {
  if (!fill) return;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(o.counter, (unsigned long long)fill);
  base = __shfl_sync(0xffffffffu, base, 0);
  for (int i = lane; i < fill; i += 32) {
    const int64_t at = (int64_t)base + i;
    if (at < o.capacity) {
      const int2 pr = st[i];
      __stcs(o.ob + o.outBase + at, pr.x);
      __stcs(o.op + o.outBase + at, pr.y);
    }
  }
}

// Stages one pair per lane that has one (all lanes of the warp call it; fill is warp-uniform).
__device__ __forceinline__ void jStage(const JOut& o, int2* st, int& fill, bool has, int b, int p, int lane) {
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if (!m) return;
  const int cnt = __popc(m);
  if (fill + cnt > kJStage) {
    __syncwarp();
    jFlush(o, st, fill, lane);
    __syncwarp();
    fill = 0;
  }
  if (has) st[fill + __popc(m & ((1u << lane) - 1u))] = make_int2(b, p);
  fill += cnt;
}

// ---- dense join: build keys in a range of at most a few times their number index a table of
// int32 build rows directly (table[key - kmin], -1 = none); duplicate keys chain through next[]
// (next[row - rowBase] = the previously inserted row with that key).  One random 4-byte lookup per
// probe row, into a table that is 4 bytes per key of the range.
__global__ void kJoinDenseBuild(ws_col_view key, int64_t base, int64_t n, int* table, long long kmin, int* next,
                                int* dup) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    long long k;
    if (!joinKeyStream(key, base + i, k)) continue;
    const int old = atomicExch(table + ((u64)k - (u64)kmin), (int)(base + i));
    next[i] = old;
    if (old >= 0) *dup = 1;
  }
}

__global__ void __launch_bounds__(kJThreads) kJoinDenseProbe(ws_col_view key, int64_t base, int64_t n,
                                                             const int* table, long long kmin, u64 range,
                                                             const int* next, int64_t rowBase, const int* dupFlag,
                                                             JOut out) {
  __shared__ int2 stage[kJWarps][kJStage];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int2* st = stage[warp];
  int fill = 0;
  const bool dup = *dupFlag != 0;
  const int64_t wstep = (int64_t)gridDim.x * kJWarps * 32 * kJPer;
  for (int64_t w0 = ((int64_t)blockIdx.x * kJWarps + warp) * 32 * kJPer; w0 < n; w0 += wstep) {
    u64 idx[kJPer];
#pragma unroll
    for (int j = 0; j < kJPer; ++j) {
      const int64_t r = w0 + j * 32 + lane;
      long long k = 0;
      const bool ok = r < n && joinKeyStream(key, base + r, k);
      idx[j] = ok ? (u64)k - (u64)kmin : range;
    }
    int b[kJPer];
#pragma unroll
    for (int j = 0; j < kJPer; ++j) b[j] = idx[j] < range ? __ldg(table + idx[j]) : -1;
#pragma unroll
    for (int j = 0; j < kJPer; ++j) {
      const bool inRange = w0 + j * 32 + lane < n;
      // an unmatched probe row of an outer join pairs with build row -1
      const bool hit = b[j] >= 0, miss = out.outer && inRange && !hit;
      if (hit && out.matched) out.matched[b[j] - out.rowBase] = 1;
      jStage(out, st, fill, hit || miss, hit ? b[j] : -1, (int)(base + w0 + j * 32 + lane), lane);
    }
    if (dup) {
      for (;;) {
        bool any = false;
#pragma unroll
        for (int j = 0; j < kJPer; ++j) {
          b[j] = b[j] >= 0 ? __ldg(next + (b[j] - rowBase)) : -1;
          any |= b[j] >= 0;
        }
        if (!__any_sync(0xffffffffu, any)) break;
#pragma unroll
        for (int j = 0; j < kJPer; ++j) {
          if (b[j] >= 0 && out.matched) out.matched[b[j] - out.rowBase] = 1;
          jStage(out, st, fill, b[j] >= 0, b[j], (int)(base + w0 + j * 32 + lane), lane);
        }
      }
    }
  }
  __syncwarp();
  jFlush(out, st, fill, lane);
}

// ---- hash join probe: each warp takes kJHashPer x 32 consecutive probe rows per step (one coalesced
// load per row slot), so each lane has kJHashPer keys, and works in rounds of independent loads: the
// keys; the first bucket of every key; the build row of every key's first matching slot; then the
// first matches are staged.  Keys with more to do (a second match in their bucket, or a full bucket
// whose run goes on) are rare; they are queued per warp and walked 32 at a time, one per lane, so the
// common path stays short and the walks run with all lanes busy.  Matches are staged per warp and
// written in coalesced runs.
struct JRest {   // a key whose probe goes on
  u64 sk;        // stored key
  u64 bucket;    // its current bucket
  int probeRow;
  unsigned m;    // slots of the current bucket that matched and are not emitted yet
  int flags;     // 1: the current bucket is full (the run goes on); 2: the key has matched
};
constexpr int kJRestCap = 64;

// Walks up to 32 queued keys, one per lane (all lanes of the warp call it; n warp-uniform, <= 32).
__device__ __forceinline__ void jWalk(const JOut& out, int2* st, int& fill, const JRest* q, int cnt, const u64* keys,
                                      const int* rows, u64 nbuckets, u64 pol, int lane) {
  const unsigned full = 0xffffffffu;
  bool live = lane < cnt;
  JRest e{};
  if (live) e = q[lane];
  u64 steps = 0;
  while (__any_sync(full, live)) {
    while (__any_sync(full, live && e.m != 0)) {
      const bool has = live && e.m != 0;
      int r = 0;
      if (has) {
        const int s = __ffs(e.m) - 1;
        e.m &= e.m - 1;
        r = __ldg(rows + e.bucket * kJRowStride + s);
        e.flags |= 2;
        if (out.matched) out.matched[r - out.rowBase] = 1;
      }
      jStage(out, st, fill, has, r, e.probeRow, lane);
    }
    bool unmatched = false;
    if (live) {
      if ((e.flags & 1) && ++steps < nbuckets) {
        e.bucket = e.bucket + 1 == nbuckets ? 0 : e.bucket + 1;
        u64 k4[4];
        ldBucket(keys + e.bucket * kJBucketWords, pol, k4);
#pragma unroll
        for (int s = 0; s < 4; ++s) e.m |= (unsigned)(k4[s] == e.sk) << s;
        e.flags = (e.flags & 2) | (k4[0] && k4[1] && k4[2] && k4[3] ? 1 : 0);
      } else {
        live = false;
        unmatched = out.outer && !(e.flags & 2);
      }
    }
    jStage(out, st, fill, unmatched, -1, e.probeRow, lane);
  }
}

__global__ void __launch_bounds__(kJThreads) kJoinProbe(ws_col_view key, int64_t base, int64_t n, JPass jp,
                                                        const u64* keys, const int* rows, u64 nbuckets, JOut out,
                                                        JFilter jf) {
  __shared__ int2 stage[kJWarps][kJStage];
  __shared__ JRest restQ[kJWarps][kJRestCap];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu, lower = (1u << lane) - 1u;
  int2* st = stage[warp];
  JRest* rq = restQ[warp];
  int fill = 0, queued = 0;  // warp-uniform
  const u64 pol = jKeepPolicy();
  const int64_t wstep = (int64_t)gridDim.x * kJWarps * 32 * kJHashPer;
  for (int64_t w0 = ((int64_t)blockIdx.x * kJWarps + warp) * 32 * kJHashPer; w0 < n; w0 += wstep) {
    u64 sk[kJHashPer], bk[kJHashPer], slot[kJHashPer][4], fb[kJHashPer], fw[kJHashPer];
    bool act[kJHashPer];
    // round 1: keys
#pragma unroll
    for (int j = 0; j < kJHashPer; ++j) {
      const int64_t r = w0 + j * 32 + lane;
      long long k = 0;
      const bool valid = r < n && joinKeyStream(key, base + r, k);
      // outer join: a NULL-key probe row matches nothing; it is emitted once, in pass 0
      if (out.outer) jStage(out, st, fill, jp.pass == 0 && r < n && !valid, -1, (int)(base + r), lane);
      const u64 h = mix64((u64)k);
      act[j] = valid && jp.mine(h);
      sk[j] = (u64)k ^ kJSign;
      bk[j] = jBucket(h, nbuckets);
      fb[j] = jFilterBits(h);
      fw[j] = jFilterWord(h, jf.mask);
    }
    // round 1b (inner joins with a key filter): keys whose filter bits are not all set have no match
    if (jf.words) {
      u64 word[kJHashPer];
#pragma unroll
      for (int j = 0; j < kJHashPer; ++j) word[j] = act[j] ? ldFilter(jf.words + fw[j], pol) : 0ull;
#pragma unroll
      for (int j = 0; j < kJHashPer; ++j) act[j] = act[j] && (word[j] & fb[j]) == fb[j];
    }
    // round 2: first buckets
#pragma unroll
    for (int j = 0; j < kJHashPer; ++j)
      if (act[j]) ldBucket(keys + bk[j] * kJBucketWords, pol, slot[j]);
    // round 3: the build row of each key's first matching slot
    unsigned m[kJHashPer];
    bool more[kJHashPer];
    int row[kJHashPer];
#pragma unroll
    for (int j = 0; j < kJHashPer; ++j) {
      m[j] = 0;
      more[j] = false;
      if (act[j]) {
#pragma unroll
        for (int q = 0; q < 4; ++q) m[j] |= (unsigned)(slot[j][q] == sk[j]) << q;
        more[j] = slot[j][0] && slot[j][1] && slot[j][2] && slot[j][3];  // full: the run may go on
      }
      row[j] = m[j] ? __ldg(rows + bk[j] * kJRowStride + (__ffs(m[j]) - 1)) : 0;
    }
    // round 4: stage the first matches (and an outer join's unmatched rows whose run ended); queue the rest
#pragma unroll
    for (int j = 0; j < kJHashPer; ++j) {
      const int pr = (int)(base + w0 + j * 32 + lane);
      const bool hit = m[j] != 0;
      if (hit && out.matched) out.matched[row[j] - out.rowBase] = 1;
      const bool unmatched = out.outer && act[j] && !hit && !more[j];
      jStage(out, st, fill, hit || unmatched, hit ? row[j] : -1, pr, lane);
      if (hit) m[j] &= m[j] - 1;
      const bool rest = m[j] != 0 || more[j];
      const unsigned rb = __ballot_sync(full, rest);
      if (!rb) continue;
      if (queued + __popc(rb) > kJRestCap) {  // walk a batch first
        __syncwarp();
        const int cnt = min(queued, 32);
        jWalk(out, st, fill, rq + queued - cnt, cnt, keys, rows, nbuckets, pol, lane);
        queued -= cnt;
        __syncwarp();
      }
      if (rest) rq[queued + __popc(rb & lower)] = JRest{sk[j], bk[j], pr, m[j], (more[j] ? 1 : 0) | (hit ? 2 : 0)};
      queued += __popc(rb);
      if (queued >= 32) {
        __syncwarp();
        jWalk(out, st, fill, rq + queued - 32, 32, keys, rows, nbuckets, pol, lane);
        queued -= 32;
        __syncwarp();
      }
    }
  }
  __syncwarp();
  while (queued > 0) {
    const int cnt = min(queued, 32);
    jWalk(out, st, fill, rq + queued - cnt, cnt, keys, rows, nbuckets, pol, lane);
    queued -= cnt;
    __syncwarp();
  }
  jFlush(out, st, fill, lane);
}

// Table budget per hash pass (bytes): the largest table that stays resident in L2 next to the streams.
int64_t joinTableBudget() {
  static const int64_t b = [] {
    const char* e = getenv("WARPSTORE_B200_JOIN_TABLE_BYTES");
    const long long v = e ? atoll(e) : 0;
    return v > 0 ? (int64_t)v : (int64_t)1 << 40;
  }();
  return b;
}



// Hash join table slots for `keys` build keys: perKey per key (default 2: load 1/2, a bucket of 4 is
// full for about 1 key in 7; the tuner may choose another), a multiple of the 4-slot bucket with at
// least one spare bucket; WARPSTORE_B200_JOIN_SLOTS_PER_KEY = 2..16 fixes the factor.
constexpr int64_t kJSlotBytes = 16;  // a 64-byte bucket of 4 slots
int64_t joinTableSlots(int64_t keys, int perKey = 0) {
  static const int64_t fixed = [] {
    const char* e = getenv("WARPSTORE_B200_JOIN_SLOTS_PER_KEY");
    const long long v = e ? atoll(e) : 0;
    return v >= 2 && v <= 16 ? (int64_t)v : (int64_t)0;
  }();
  const int64_t per = fixed ? fixed : perKey >= 2 ? perKey : 2;
  return ((per * keys + 3) / 4 + 1) * 4;
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
  if (ncols < 0 || ncols > WS_MAX_COLS || nb < 0) throw Error("select: bad column or batch count", WS_ERR_ARG);
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

}  // extern "C"

namespace ws {
namespace {

// Pairs (b, -1) for every build row with matched[b] == 0 (ascending), after `m` pairs of the output.
__global__ void kUnmatchedCount(const uint8_t* matched, int64_t n, int64_t* counts) {
  __shared__ int wsum[8];
  const int64_t i0 = (int64_t)blockIdx.x * 1024 + threadIdx.x * 4;
  int c = 0;
  for (int i = 0; i < 4; ++i) c += i0 + i < n && !matched[i0 + i];
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += wsum[w];
    counts[blockIdx.x] = t;
  }
}
__global__ void kUnmatchedWrite(const uint8_t* matched, int64_t n, const int64_t* offs, int64_t m, int32_t* ob,
                                int32_t* op) {
  __shared__ int wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * 1024 + threadIdx.x * 4;
  int c = 0;
  for (int i = 0; i < 4; ++i) c += i0 + i < n && !matched[i0 + i];
  int incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  int64_t at = m + offs[blockIdx.x] + before + incl - c;
  for (int i = 0; i < 4; ++i)
    if (i0 + i < n && !matched[i0 + i]) ob[at] = (int32_t)(i0 + i), op[at] = -1, ++at;
}
// Every probe row of [base, base + n) paired with build row -1 (outer join, no build key at all).
__global__ void kAllUnmatched(int64_t base, int64_t n, int32_t* ob, int32_t* op, unsigned long long* counter) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    ob[j] = -1, op[j] = (int32_t)(base + j);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(counter, (unsigned long long)n);
}
__global__ void kCross(int64_t na, int64_t nb, int32_t* oa, int32_t* ob) {
  const int64_t n = na * nb;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    oa[i] = (int32_t)(i / nb);
    ob[i] = (int32_t)(i % nb);
  }
}

}  // namespace

// The autotuner's choice of slots per build key for a one-pass hash join of one build and one probe
// partition (keys: non-NULL build keys): the recorded one, or in tuning mode the fastest of 2, 3 and 4,
// each timed (best of two) building its table and probing every row into scratch pair buffers.
// 0: the default.
static int joinSlotsChoice(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int64_t keys) {
  int lb = 0, lp = 0;
  while (lb < 62 && ((int64_t)1 << (lb + 1)) <= keys) ++lb;
  while (lp < 62 && ((int64_t)1 << (lp + 1)) <= np) ++lp;
  const std::string key = "join:b" + std::to_string(lb) + ":p" + std::to_string(lp);
  TuneChoice c;
  if (tuneLookup(key, c)) return c.slotsPerKey;
  if (tuneMode() != WS_TUNE_ON || np > INT32_MAX) return 0;
  const int64_t maxC = joinTableSlots(keys, 4);
  DBuf<u64> table(maxC / 4 * kJBucketWords);
  DBuf<int> flags(1);
  DBuf<int32_t> ob(std::max<int64_t>(np, 1)), op(std::max<int64_t>(np, 1));
  DBuf<unsigned long long> ctr(1);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WS_CK(cudaEventCreate(&e0));
  WS_CK(cudaEventCreate(&e1));
  int best = 0;
  double bestMs = 1e300;
  try {
    for (int per : {2, 3, 4}) {
      const int64_t cs = joinTableSlots(keys, per);
      double ms = 1e300;
      int full = 0;
      for (int rep = 0; rep < 2; ++rep) {
        WS_CK(cudaEventRecord(e0, stream()));
        WS_CK(cudaMemsetAsync(table.p, 0, 8 * kJBucketWords * (cs / 4), stream()));
        WS_CK(cudaMemsetAsync(flags.p, 0, 4, stream()));
        WS_CK(cudaMemsetAsync(ctr.p, 0, 8, stream()));
        WS_LAUNCH(kJoinBuild, gridFor(nb), 256, 0, build_key, (int64_t)0, nb, JPass{0, 0}, table.p,
                  (int*)(table.p + 4), (u64)(cs / 4), flags.p, JFilter{nullptr, 0});
        const JOut jo{ob.p, op.p, 0, np, ctr.p, 0, nullptr, 0};
        WS_LAUNCH(kJoinProbe, gridFor((np + kJHashPer - 1) / kJHashPer, kJThreads), kJThreads, 0, probe_key,
                  (int64_t)0, np, JPass{0, 0}, table.p, (const int*)(table.p + 4), (u64)(cs / 4), jo,
                  JFilter{nullptr, 0});
        WS_CK(cudaEventRecord(e1, stream()));
        WS_CK(cudaEventSynchronize(e1));
        float t = 0;
        WS_CK(cudaEventElapsedTime(&t, e0, e1));
        ms = std::min(ms, (double)t);
      }
      d2hSync(&full, flags.p, 4);
      if (!full && ms < bestMs) bestMs = ms, best = per;
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!best) return 0;
  TuneChoice t;
  t.slotsPerKey = best;
  tuneStore(key, t, bestMs * 1000);
  return best;
}

// Inner (outer = 0) or outer equi join over build / probe partitions; see ws_hash_join_parts and
// ws_hash_join_outer.  full: also the build rows that matched nothing, paired with probe row -1.
// firstCap > 0 (an inner join of one partition): the pair buffers' capacity of the first attempt
// instead of the probe rows.  keyFilter: the caller expects most probe rows to find no match (see
// JFilter).  Returns the attempts made (a second one when the first capacity was short).
static int joinImpl(ws_col_view build_key, const int64_t* boff, int pb, ws_col_view probe_key, const int64_t* poff,
                    int pp, int outer, bool full, int32_t** out_build, int32_t** out_probe, int64_t* out_off,
                    int64_t* m_out, int64_t firstCap = 0, bool keyFilter = false) {
  {
    *out_build = *out_probe = nullptr;
    if (pb < 1 || pp < 1 || (pb != 1 && pb != pp)) throw Error("internal: partition count mismatch in join", WS_ERR_INTERNAL);
    const int64_t nb = boff[pb], np = poff[pp];
    if (out_off)
      for (int p = 0; p <= pp; ++p) out_off[p] = 0;
    *m_out = 0;
    if (nb == 0 || np == 0) {
      // inner: nothing; outer: every probe row unmatched; full: every build row too
      const int64_t m = outer ? np + (full ? nb : 0) : 0;
      if (m > INT32_MAX) throw Error("join result too large (>2^31 rows)", WS_ERR_INTERNAL);
      DBuf<int32_t> ob(std::max<int64_t>(m, 1)), op(std::max<int64_t>(m, 1));
      DBuf<unsigned long long> ctr(1);
      if (outer && np) WS_LAUNCH(kAllUnmatched, gridFor(np), 256, 0, (int64_t)0, np, ob.p, op.p, ctr.p);
      if (outer && full && nb) WS_LAUNCH(kAllUnmatched, gridFor(nb), 256, 0, (int64_t)0, nb, op.p + np, ob.p + np, ctr.p);
      if (out_off)
        for (int p = 0; p <= pp; ++p) out_off[p] = outer ? poff[p] : 0;
      *out_build = ob.release();
      *out_probe = op.release();
      *m_out = m;
      return 1;
    }
    DBuf<uint8_t> matchedBuf(full ? nb : 1);
    uint8_t* matched = full ? matchedBuf.p : nullptr;
    if (full) WS_CK(cudaMemsetAsync(matched, 0, nb, stream()));
    // Hash passes per build partition (2^bits) from its row count and the table budget.
    std::vector<int> bits(pb, 0);
    for (int q = 0; q < pb; ++q) {
      const int64_t nq = boff[q + 1] - boff[q];
      const int64_t npq = pb == 1 ? np : poff[q + 1] - poff[q];  // probe rows joined with build partition q
      (void)npq;
      while (bits[q] < 6 && joinTableSlots((nq >> bits[q]) + 1) * kJSlotBytes > joinTableBudget()) ++bits[q];
    }
    // Build-key statistics (non-NULL count, min, max, keys per hash pass) of every partition.
    DBuf<unsigned long long> stats((int64_t)pb * kJStatWords);
    for (int q = 0; q < pb; ++q) {
      const int64_t n = boff[q + 1] - boff[q];
      WS_LAUNCH(kJoinStatsInit, 1, 128, 0, stats.p + (int64_t)q * kJStatWords);
      if (n) WS_LAUNCH(kJoinStats, gridFor(n), 256, 0, build_key, boff[q], n, bits[q], stats.p + (int64_t)q * kJStatWords);
    }
    std::vector<unsigned long long> hs((size_t)pb * kJStatWords);
    WS_CK(cudaMemcpyAsync(hs.data(), stats.p, 8 * hs.size(), cudaMemcpyDeviceToHost, stream()));
    sync();
    // Per partition: dense (key range <= max(4 x keys, 2^16), below 2^31) or hash passes.
    std::vector<char> dense(pb, 0);
    std::vector<long long> kmin(pb, 0);
    std::vector<u64> range(pb, 0);
    std::vector<std::vector<int64_t>> cap(pb);
    int64_t denseSlots = 1, nextRows = 1, tableSlots = 2;
    for (int q = 0; q < pb; ++q) {
      const unsigned long long* st = hs.data() + (size_t)q * kJStatWords;
      const int64_t keys = (int64_t)st[0];
      if (!keys) continue;
      kmin[q] = (long long)st[1];
      range[q] = (u64)(long long)st[2] - (u64)(long long)st[1] + 1;  // 0 when the keys span all of int64
      if (range[q] && range[q] < ((u64)1 << 31) && range[q] <= std::max<u64>(4 * (u64)keys, 1 << 16)) {
        dense[q] = 1;
        denseSlots = std::max<int64_t>(denseSlots, (int64_t)range[q]);
        nextRows = std::max<int64_t>(nextRows, boff[q + 1] - boff[q]);
        continue;
      }
      for (int p = 0; p < (1 << bits[q]); ++p) {
        const int64_t c = joinTableSlots(bits[q] ? (int64_t)st[3 + p] : keys);
        cap[q].push_back(c);
        tableSlots = std::max(tableSlots, c);
      }
    }
    // the tuner's table size for a one-pass hash join of one partition a side
    if (pb == 1 && pp == 1 && boff[0] == 0 && poff[0] == 0 && !dense[0] && cap[0].size() == 1 && !bits[0]) {
      const int per = joinSlotsChoice(build_key, nb, probe_key, np, (int64_t)hs[0]);
      if (per) {
        cap[0][0] = joinTableSlots((int64_t)hs[0], per);
        tableSlots = std::max(tableSlots, cap[0][0]);
      }
    }
    bool anyDense = false, anyHash = false;
    for (int q = 0; q < pb; ++q) anyDense |= dense[q] != 0, anyHash |= !cap[q].empty();
    // one table of 64-byte buckets (keys, then rows: kJBucketWords)
    DBuf<u64> table(anyHash ? tableSlots / 4 * kJBucketWords : kJBucketWords);
    u64* tkeys = table.p;
    int* trows = (int*)(table.p + 4);
    DBuf<int> dtable(anyDense ? denseSlots : 1), next(anyDense ? nextRows : 1);
    // Key filters (JFilter) for the hash-built partitions of an inner join built in one pass, 16 bits
    // per build key, when the caller expects few probe rows to match (keyFilter) and the table has 2^20
    // keys or more (L2 does not hold it, so a probe that finds no match costs a random DRAM access).
    // Measured (7.5M build keys x 60M probe rows): a quarter of the probes matching 3.13 -> 2.54 ms (15M
    // keys), half 1.70 -> 1.68 ms, all 1.88 -> 2.21 ms.  WARPSTORE_B200_JOIN_FILTER = 0 never, 1 always.
    static const int filterMode = [] {
      const char* e = getenv("WARPSTORE_B200_JOIN_FILTER");
      return e && *e ? atoi(e) : -1;
    }();
    std::vector<u64> filterWords(pb, 0);
    u64 maxFilterWords = 0;
    for (int q = 0; q < pb; ++q) {
      const int64_t keys = (int64_t)hs[(size_t)q * kJStatWords];
      if (outer || dense[q] || cap[q].empty() || bits[q] || filterMode == 0) continue;
      if (filterMode != 1 && (!keyFilter || keys < ((int64_t)1 << 20))) continue;
      u64 w = 1024;
      while ((int64_t)w < keys / 4) w <<= 1;
      filterWords[q] = w;
      maxFilterWords = std::max(maxFilterWords, w);
    }
    DBuf<u64> filter(maxFilterWords ? (int64_t)maxFilterWords : 1);
    DBuf<int> flags(2);  // [0] hash table full, [1] duplicate dense keys
    WS_CK(cudaMemsetAsync(flags.p, 0, 8, stream()));
    // One probe pass with output capacity = probe rows per partition (enough for every join whose
    // build keys are unique); if a partition produced more, a second pass writes with exact sizes.
    std::vector<int64_t> capOut(pp), outStart(pp + 1, 0);
    for (int p = 0; p < pp; ++p) {
      capOut[p] = poff[p + 1] - poff[p];
      if (firstCap > 0 && !outer && pp == 1) capOut[p] = std::min<int64_t>(firstCap, INT32_MAX);
      outStart[p + 1] = outStart[p] + capOut[p];
    }
    DBuf<unsigned long long> counters(pp);
    std::vector<unsigned long long> cnt(pp);
    for (int attempt = 0; attempt < 2; ++attempt) {
      WS_CK(cudaMemsetAsync(counters.p, 0, 8 * pp, stream()));
      DBuf<int32_t> ob(std::max<int64_t>(outStart[pp], 1)), op(std::max<int64_t>(outStart[pp], 1));
      for (int q = 0; q < pb; ++q) {
        const int64_t nbq = boff[q + 1] - boff[q];
        const int npass = dense[q] ? 1 : (int)cap[q].size();  // 0: no non-NULL build key
        if (npass == 0 && outer)
          for (int p = 0; p < pp; ++p) {
            if (pb != 1 && p != q) continue;
            const int64_t n = poff[p + 1] - poff[p];
            if (n && n <= capOut[p])
              WS_LAUNCH(kAllUnmatched, gridFor(n), 256, 0, poff[p], n, ob.p + outStart[p], op.p + outStart[p],
                        counters.p + p);
          }
        for (int pass = 0; pass < npass; ++pass) {
          const JPass jp{bits[q], pass};
          const int64_t c = dense[q] ? 0 : cap[q][pass];
          const JFilter jf{filterWords[q] ? filter.p : nullptr, filterWords[q] ? filterWords[q] - 1 : 0};
          if (dense[q]) {
            WS_CK(cudaMemsetAsync(dtable.p, 0xff, 4 * range[q], stream()));
            WS_CK(cudaMemsetAsync(flags.p + 1, 0, 4, stream()));
            WS_LAUNCH(kJoinDenseBuild, gridFor(nbq), 256, 0, build_key, boff[q], nbq, dtable.p, kmin[q], next.p,
                      flags.p + 1);
          } else {
            WS_CK(cudaMemsetAsync(tkeys, 0, 8 * kJBucketWords * (c / 4), stream()));
            if (jf.words) WS_CK(cudaMemsetAsync(jf.words, 0, 8 * filterWords[q], stream()));
            WS_LAUNCH(kJoinBuild, gridFor(nbq), 256, 0, build_key, boff[q], nbq, jp, tkeys, trows, (u64)(c / 4),
                      flags.p, jf);
          }
          for (int p = 0; p < pp; ++p) {  // probe partitions joined with build partition q
            if (pb != 1 && p != q) continue;
            const int64_t n = poff[p + 1] - poff[p];
            if (!n) continue;
            const JOut jo{ob.p, op.p, outStart[p], capOut[p], counters.p + p, outer, matched, boff[q]};
            const int grid = gridFor((n + kJPer - 1) / kJPer, kJThreads);
            const int hgrid = gridFor((n + kJHashPer - 1) / kJHashPer, kJThreads);
            if (dense[q])
              WS_LAUNCH(kJoinDenseProbe, grid, kJThreads, 0, probe_key, poff[p], n, dtable.p, kmin[q], range[q], next.p,
                        boff[q], flags.p + 1, jo);
            else
              WS_LAUNCH(kJoinProbe, hgrid, kJThreads, 0, probe_key, poff[p], n, jp, tkeys, trows, (u64)(c / 4), jo,
                        jf);
          }
        }
      }
      int e = 0;
      WS_CK(cudaMemcpyAsync(cnt.data(), counters.p, 8 * pp, cudaMemcpyDeviceToHost, stream()));
      WS_CK(cudaMemcpyAsync(&e, flags.p, 4, cudaMemcpyDeviceToHost, stream()));
      sync();
      if (e) throw Error("internal: join hash table full", WS_ERR_INTERNAL);
      bool fits = true;
      int64_t m = 0;
      for (int p = 0; p < pp; ++p) {
        fits &= (int64_t)cnt[p] <= capOut[p];
        m += (int64_t)cnt[p];
      }
      if (m > INT32_MAX) throw Error("join result too large (>2^31 rows)", WS_ERR_INTERNAL);
      if (fits && full) {  // single partition: append the build rows that matched nothing
        const int64_t nchunks = (nb + 1023) / 1024;
        DBuf<int64_t> counts(nchunks + 1);
        WS_LAUNCH(kUnmatchedCount, (unsigned)nchunks, 256, 0, matched, nb, counts.p);
        WS_LAUNCH(kScanTiles, 1, 1024, 0, counts.p, nchunks);
        int64_t extra = 0;
        d2hSync(&extra, counts.p + nchunks, 8);
        if (m + extra > INT32_MAX) throw Error("join result too large (>2^31 rows)", WS_ERR_INTERNAL);
        DBuf<int32_t> cb(std::max<int64_t>(m + extra, 1)), cp(std::max<int64_t>(m + extra, 1));
        if (m) {
          WS_CK(cudaMemcpyAsync(cb.p, ob.p, 4 * m, cudaMemcpyDeviceToDevice, stream()));
          WS_CK(cudaMemcpyAsync(cp.p, op.p, 4 * m, cudaMemcpyDeviceToDevice, stream()));
        }
        if (extra) WS_LAUNCH(kUnmatchedWrite, (unsigned)nchunks, 256, 0, matched, nb, counts.p, m, cb.p, cp.p);
        *out_build = cb.release();
        *out_probe = cp.release();
        *m_out = m + extra;
        return attempt + 1;
      }
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
        return attempt + 1;
      }
      for (int p = 0; p < pp; ++p) {  // exact sizes for the second attempt
        capOut[p] = (int64_t)cnt[p];
        outStart[p + 1] = outStart[p] + capOut[p];
      }
    }
    throw Error("internal: join output sizing failed", WS_ERR_INTERNAL);
  }
}

}  // namespace ws

extern "C" {

int ws_hash_join_parts(ws_col_view build_key, const int64_t* boff, int nbparts, ws_col_view probe_key,
                       const int64_t* poff, int npparts, int32_t** out_build, int32_t** out_probe, int64_t* out_off,
                       int64_t* m_out) {
  return guardedCall([&] {
    joinImpl(build_key, boff, nbparts, probe_key, poff, npparts, 0, false, out_build, out_probe, out_off, m_out);
  });
}

int ws_hash_join(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int32_t** out_build,
                 int32_t** out_probe, int64_t* m) {
  const int64_t bo[2] = {0, nb}, po[2] = {0, np};
  return ws_hash_join_parts(build_key, bo, 1, probe_key, po, 1, out_build, out_probe, nullptr, m);
}

int ws_hash_join_sized(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int64_t first_capacity,
                       int32_t** out_build, int32_t** out_probe, int64_t* m, int* attempts) {
  return guardedCall([&] {
    const int64_t bo[2] = {0, nb}, po[2] = {0, np};
    // a first capacity well below the probe rows says that most probe rows find no match (pairs are at
    // least the matching probe rows): the key filter pays there
    const int a = joinImpl(build_key, bo, 1, probe_key, po, 1, 0, false, out_build, out_probe, nullptr, m,
                           std::max<int64_t>(first_capacity, 1), (double)first_capacity < 0.35 * (double)np);
    if (attempts) *attempts = a;
  });
}

int ws_hash_join_outer(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int full,
                       int32_t** out_build, int32_t** out_probe, int64_t* m) {
  return guardedCall([&] {
    const int64_t bo[2] = {0, nb}, po[2] = {0, np};
    joinImpl(build_key, bo, 1, probe_key, po, 1, 1, full != 0, out_build, out_probe, nullptr, m);
  });
}

int ws_join_key_sample(ws_col_view key, int64_t n, uint64_t tau, uint64_t* out, int64_t cap, int64_t* count) {
  return guardedCall([&] {
    *count = 0;
    if (n < 0 || cap < 0) throw Error("join key sample: negative size", WS_ERR_ARG);
    if (n == 0) return;
    DBuf<unsigned long long> c(1);
    DBuf<u64> d(std::max<int64_t>(cap, 1));
    WS_CK(cudaMemsetAsync(c.p, 0, 8, stream()));
    WS_LAUNCH(kJoinKeySample, gridFor(n), 256, 0, key, n, (u64)tau, d.p, cap, c.p);
    unsigned long long hc = 0;
    WS_CK(cudaMemcpyAsync(&hc, c.p, 8, cudaMemcpyDeviceToHost, stream()));
    sync();
    *count = (int64_t)hc;
    const int64_t got = std::min<int64_t>((int64_t)hc, cap);
    if (got) {
      WS_CK(cudaMemcpyAsync(out, d.p, 8 * (size_t)got, cudaMemcpyDeviceToHost, stream()));
      sync();
    }
  });
}

int ws_cross_join(int64_t na, int64_t nb, int32_t** out_a, int32_t** out_b, int64_t* m) {
  return guardedCall([&] {
    *out_a = *out_b = nullptr;
    const int64_t n = na * nb;
    if (na < 0 || nb < 0) throw Error("negative row count", WS_ERR_ARG);
    if (n > 200000000)
      throw Error("cross join too large (" + std::to_string(n) + " rows); add a join condition", WS_ERR_INTERNAL);
    DBuf<int32_t> a(std::max<int64_t>(n, 1)), b(std::max<int64_t>(n, 1));
    if (n) WS_LAUNCH(kCross, gridFor(n), 256, 0, na, nb, a.p, b.p);
    *out_a = a.release();
    *out_b = b.release();
    *m = n;
  });
}

}  // extern "C"
