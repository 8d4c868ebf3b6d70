// Scan kernel bodies, templated over a row evaluator `Ev`.  The library instantiates them with the
// on-device interpreter (InterpEv, ws_interp.cuh); every query plan instantiates them again with its
// own generated evaluator, compiled by NVRTC for sm_100a (ws_codegen.cpp).  No host headers.
//
// Evaluator contract (all row indices are within the current batch):
//   static constexpr int NK, NA;            loop bounds (>= nk(), na())
//   Ev(const Launch&);  void bind(const Launch&, int batch);  bool fastOk;
//   int nk(), na(), rowWords(), kind(a), woff(a); bool keyInt(k);
//   void load(i64 r0, bool fast, int nv);   rows r0 .. r0+3 (nv valid) into registers
//   bool where(i); i64 ikey(k, i); double dkey(k, i); bool ival(a, i, i64&); double dval(a, i)
//   void prep(i, bool live); void finish()
//
// Work decomposition: a batch (segment / write buffer) is cut into tiles of kTile rows; a CTA of
// kThreads threads takes one tile per iteration, each thread 4 consecutive rows (128-bit loads of
// 4-byte columns, 2 x 128-bit of 8-byte columns).  Grids are persistent (a multiple of the SM count);
// CTAs stride over the tiles of all batches of the launch.
#pragma once
#include "ws_dev.cuh"

namespace ws {

constexpr int kThreads = 256;
constexpr int kTile = kThreads * 4;
constexpr u64 kEmpty = ~0ull;
constexpr int kMaxRowWords = 1 + 2 * WS_MAX_AGGS;

WS_DI u64 mix64(u64 x) {  // splitmix64 finalizer (Steele, Lea, Flood 2014)
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// The 4 loaded rows of a thread, one after another: filter the row, evaluate its common
// subexpressions (prep), hand it to f when it passes.  Evaluating and consuming each row before the
// next keeps one row's temporaries live at a time (fewer registers, more resident warps).
template <class Ev, class F>
WS_DI void rowGroup(Ev& ev, unsigned live, int b, i64 r0, F&& f) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const bool ok = ((live >> i) & 1u) && ev.where(i);
    ev.prep(i, ok);
    if (ok) f(i, b, r0 + i);
  }
}

// The batch holding tile t of the launch (tileStart[b] <= t < tileStart[b + 1]; empty batches skipped).
WS_DI int batchOfTile(const Launch& L, i64 t) {
  int lo = 0, hi = L.nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(L.tileStart + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Walks the tiles this CTA owns: the contiguous range [T c / G, T (c + 1) / G) of the launch's T tiles
// (c = ctaIndex, G = ctaCount), batch by batch.  A CTA crosses one or two batches, so the batch's
// size, bitmap and column views (and an encoded column's header) are read once or twice per CTA
// rather than once per batch of the launch.  tile(t, b, r0, n, del) is called by every thread of the
// CTA for each tile t of batch b (r0 = the thread's first row in the batch, n = the batch's rows,
// del = its deleted bitmap); it returns true to end the walk (the same value in every thread).
template <class Ev, class F>
WS_DI void forEachOwnedTile(const Launch& L, Ev& ev, F&& tile) {
  const i64 T = L.ntiles, G = ctaCount(L), c = ctaIndex(L);
  i64 t = T * c / G;
  const i64 tEnd = T * (c + 1) / G;
  if (t >= tEnd) return;
  for (int b = batchOfTile(L, t); t < tEnd && b < L.nb; ++b) {
    const i64 bs = __ldg(L.tileStart + b), bend = __ldg(L.tileStart + b + 1), be = bend < tEnd ? bend : tEnd;
    if (t >= be) continue;  // an empty batch
    ev.bind(L, b);
    const i64 n = __ldg(L.n + b);
    const uint32_t* del = L.del[b];
    for (; t < be; ++t)
      if (tile(t, b, (t - bs) * kTile + threadIdx.x * 4, n, del)) return;
  }
}

// Loads the thread's 4 rows from r0 and visits the live ones (not deleted, passing the filter).
template <class Ev, class F>
WS_DI void visitRows(Ev& ev, int b, i64 r0, i64 n, const uint32_t* del, F&& f) {
  const i64 left = n - r0;
  if (left <= 0) return;
  const int nv = left >= 4 ? 4 : (int)left;
  ev.load(r0, ev.fastOk && nv == 4, nv);
  unsigned live = (1u << nv) - 1;
  if (del) live &= ~(__ldg(del + (r0 >> 5)) >> (r0 & 31)) & 0xfu;
  rowGroup(ev, live, b, r0, f);
}

// Visits every live row of the tiles this CTA owns.  f(i, batch, row) is called with i = the row's
// position (0..3) in the evaluator's 4-row group.  tileEnd() is called by every thread of the CTA
// after each of the CTA's tiles (a CTA-uniform point); it returns the same value in every thread,
// true to end the visit there.
template <class Ev, class F, class E>
WS_DI void forEachRowTiles(const Launch& L, Ev& ev, F&& f, E&& tileEnd) {
  forEachOwnedTile(L, ev, [&](i64, int b, i64 r0, i64 n, const uint32_t* del) {
    visitRows(ev, b, r0, n, del, f);
    return tileEnd();
  });
  ev.finish();
}

template <class Ev, class F>
WS_DI void forEachRow(const Launch& L, Ev& ev, F&& f) {
  forEachOwnedTile(L, ev, [&](i64, int b, i64 r0, i64 n, const uint32_t* del) {
    visitRows(ev, b, r0, n, del, f);
    return false;
  });
  ev.finish();
}

// Same visit, with each tile's column chunks brought into shared memory by bulk asynchronous copies
// (TMA engine), warp-specialized: the CTA has kThreads consumer threads plus one producer warp (the
// last).  A ring of S stages of Ev::STAGE_BYTES has two mbarriers per stage: `full` (the producer's
// arrive.expect_tx; the copies complete its transaction count) and `empty` (one arrival per consumer
// warp once it has read the stage).  The producer refills a stage as soon as every consumer warp has
// released it, so consumers never wait on a CTA-wide barrier.  Tiles that cannot be copied in bulk (a
// batch's ragged last tile, a column not 16-byte aligned) are marked "direct": their full barrier gets
// a plain arrive and the consumers read global memory as forEachRow does.  Every wait is bounded
// (2^L.waitLog2 cycles); one that runs out sets err[2] and ends that warp's loop.  Before the producer
// warp leaves, it waits (bounded, ~2 s) until the copies of the stages it issued last have landed, so
// no bulk copy is still writing into the CTA's shared memory when the CTA ends.
constexpr int kStagedThreads = kThreads + 32;

template <class Ev, class F>
WS_DI void forEachRowStaged(const Launch& L, Ev& ev, unsigned char* stages, int S, F&& f) {
  __shared__ __align__(8) u64 full[8], empty[8];
  __shared__ int smode[8];
  __shared__ typename Ev::Stage pst;  // the producer's view of its current batch
  constexpr int kConsumerWarps = kThreads / 32;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbarInit(smemAddr(&full[s]), 1);
      mbarInit(smemAddr(&empty[s]), kConsumerWarps);
    }
    fenceMbarInit();
    fenceProxyAsync();
  }
  __syncthreads();
  // this CTA's tiles: the contiguous range [tFirst, tFirst + K) (as forEachOwnedTile)
  const i64 tFirst = L.ntiles * (i64)ctaIndex(L) / ctaCount(L);
  const i64 K = L.ntiles * ((i64)ctaIndex(L) + 1) / ctaCount(L) - tFirst;
  if (warp == kConsumerWarps) {  // ---- producer warp (one elected lane)
    if (lane == 0) {
      int pb = K > 0 ? batchOfTile(L, tFirst) : 0, pbatch = -1;
      i64 issued = 0;
      for (i64 k = 0; k < K; ++k) {
        const int s = (int)(k % S);
        if (k >= S && !mbarWait(smemAddr(&empty[s]), (unsigned)(((k / S) - 1) & 1), L.waitLog2)) {
          L.err[2] = 1;
          break;
        }
        issued = k + 1;
        const i64 t = tFirst + k;
        while (t >= __ldg(L.tileStart + pb + 1)) ++pb;
        if (pb != pbatch) {
          Ev::stageBind(L, pb, pst);
          pbatch = pb;
        }
        const i64 tr0 = (t - __ldg(L.tileStart + pb)) * kTile;
        const bool bulk = pst.ok && tr0 + kTile <= __ldg(L.n + pb);
        smode[s] = bulk;
        const unsigned bar = smemAddr(&full[s]);
        if (bulk) {
          fenceProxyAsync();  // the stage was last read through the generic proxy
          mbarArriveTx(bar, pst.bytes);
          Ev::stageIssue(pst, tr0, smemAddr(stages + (size_t)s * Ev::STAGE_BYTES), bar);
        } else {
          mbarArrive(bar);
        }
      }
      // drain: the last phase issued on each stage completes when its copies have landed (earlier
      // phases completed before their stage was reissued)
      for (i64 k = issued > S ? issued - S : 0; k < issued; ++k)
        if (!mbarWait(smemAddr(&full[(int)(k % S)]), (unsigned)((k / S) & 1))) L.err[2] = 1;
    }
    __syncwarp();
    return;
  }
  // ---- consumer warps
  int b = K > 0 ? batchOfTile(L, tFirst) : 0, bound = -1;
  for (i64 k = 0; k < K; ++k) {
    const i64 t = tFirst + k;
    const int s = (int)(k % S);
    if (!__all_sync(0xffffffffu, mbarWait(smemAddr(&full[s]), (unsigned)((k / S) & 1), L.waitLog2))) {
      if (lane == 0) L.err[2] = 1;
      break;
    }
    while (t >= __ldg(L.tileStart + b + 1)) ++b;
    if (b != bound) {
      ev.bind(L, b);
      bound = b;
    }
    const i64 n = __ldg(L.n + b);
    const i64 r0 = (t - __ldg(L.tileStart + b)) * kTile + tid * 4;
    const i64 left = n - r0;
    if (left > 0) {
      const int nv = left >= 4 ? 4 : (int)left;
      if (smode[s]) ev.loadStage(stages + (size_t)s * Ev::STAGE_BYTES, tid * 4);
      else ev.load(r0, ev.fastOk && nv == 4, nv);
      unsigned live = (1u << nv) - 1;
      const uint32_t* del = L.del[b];
      if (del) live &= ~(__ldg(del + (r0 >> 5)) >> (r0 & 31)) & 0xfu;
      rowGroup(ev, live, b, r0, f);
    }
    __syncwarp();
    if (lane == 0) mbarArrive(smemAddr(&empty[s]));  // this warp is done with the stage
  }
  ev.finish();
}

// Visits rows, staged through shared memory when the evaluator supports it and stages were given.
template <class Ev, class F>
WS_DI void scanRows(const Launch& L, Ev& ev, F&& f) {
  if constexpr (Ev::STAGED) {
    if (L.stages >= 2 && blockDim.x == kStagedThreads) {
      extern __shared__ __align__(16) u64 wsSmem[];
      forEachRowStaged(L, ev, (unsigned char*)wsSmem, L.stages, f);
      return;
    }
  }
  forEachRow(L, ev, f);
}

// ------------------------------------------------------------------ register rows
// Per-thread accumulators of the no-key and dense kernels: one word per slot (fwoff).  An integer SUM
// adds into an int64 word; when an addition overflows it (signed), the word keeps the wrapped value
// and +-1 goes to the high word of the CTA's shared int128 spill counter of its (group, slot), so the
// exact sum is word + 2^64 * spill at the end.
template <class Ev>
WS_DI void fastIdentity(const Ev& ev, u64* w) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.fwoff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: case SK_ISUM: case SK_DSUM: w[o] = 0; break;
      case SK_IMIN: w[o] = (u64)0x7fffffffffffffffll; break;
      case SK_IMAX: w[o] = (u64)0x8000000000000000ll; break;
      case SK_DMIN: w[o] = (u64)dord(__longlong_as_double(0x7ff0000000000000ll)); break;
      case SK_DMAX: w[o] = (u64)dord(__longlong_as_double((i64)0xfff0000000000000ull)); break;
      default: break;
    }
  }
}
// The register-row contribution of row i (NULL arguments: the slot's identity).
template <class Ev>
WS_DI void fastOfInput(const Ev& ev, int i, u64* x) {
  fastIdentity(ev, x);
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.fwoff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: x[o] = 1; break;
      case SK_ISUM: case SK_IMIN: case SK_IMAX: {
        i64 v;
        if (ev.ival(a, i, v)) x[o] = (u64)v;
        break;
      }
      case SK_DSUM: {
        const double v = ev.dval(a, i);
        if (v == v) x[o] = (u64)__double_as_longlong(v);
        break;
      }
      case SK_DMIN: case SK_DMAX: {
        const double v = ev.dval(a, i);
        if (v == v) x[o] = (u64)dord(v);
        break;
      }
      default: break;
    }
  }
}
// *w += x for an int64 SUM word, carrying a signed overflow into the spill's high word.
WS_DI void addCarry(u64* w, u64 x, u64* spillHi) {
  const u64 old = *w, r = old + x;
  const unsigned ho = (unsigned)(old >> 32), hx = (unsigned)(x >> 32), hr = (unsigned)(r >> 32);
  if ((int)((ho ^ hr) & (hx ^ hr)) < 0) atomicAdd(spillHi, (int)hx < 0 ? ~0ull : 1ull);  // signed overflow
  *w = r;
}
// Exact integer sums without a test per addition.  A thread adds at most R rows into any one of its
// integer SUM words.  While every argument x has |x| <= 2^(63 - k), with 2^k >= R, no partial sum of
// those additions leaves the int64 range, so the words need no overflow test.  The host sets
// L.sumShift = 31 - k for each launch (-1 when no k applies).  sumMagnitude ORs the high words of the
// row's SUM arguments' magnitudes (x >= 0: x >> 32; x < 0: ~x >> 32 = (|x| - 1) >> 32); the bound holds
// while (magnitude >> sumShift) == 0.  A thread that meets a row breaking it switches to tested
// additions (signed overflow carried into the int128 spill) for the rest of the launch, so words that
// take unbounded values are always tested from their first such value on.
template <class Ev>
WS_DI unsigned sumMagnitude(const Ev& ev, const u64* x) {
  unsigned m = 0;
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    if (ev.kind(a) == SK_ISUM) {
      const unsigned hi = (unsigned)(x[ev.fwoff(a)] >> 32);
      m |= hi ^ (unsigned)((int)hi >> 31);
    }
  }
  return m;
}
WS_DI bool sumsNeedTests(const Launch& L, unsigned magnitude) {
  return L.sumShift < 0 || (magnitude >> L.sumShift) != 0;
}

// w += x (register rows); spill = this group's [slot][2] int128 counters
template <class Ev>
WS_DI void fastCombine(const Ev& ev, u64* w, const u64* x, u64* spill) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.fwoff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: w[o] += x[o]; break;
      case SK_ISUM: addCarry(&w[o], x[o], spill + 2 * a + 1); break;
      case SK_IMIN: case SK_DMIN: if ((i64)x[o] < (i64)w[o]) w[o] = x[o]; break;
      case SK_IMAX: case SK_DMAX: if ((i64)x[o] > (i64)w[o]) w[o] = x[o]; break;
      case SK_DSUM:
        w[o] = (u64)__double_as_longlong(__longlong_as_double((i64)w[o]) + __longlong_as_double((i64)x[o]));
        break;
      default: break;
    }
  }
}
// register row -> accumulator row (integer sums widened to int128)
template <class Ev>
WS_DI void fastExpand(const Ev& ev, const u64* f, u64* w) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.woff(a), fo = ev.fwoff(a);
    if (ev.kind(a) == SK_ISUM) w[o] = f[fo], w[o + 1] = (u64)((i64)f[fo] >> 63);
    else if (ev.kind(a) != SK_NONE) w[o] = f[fo];
  }
}

// ------------------------------------------------------------------ row words
// A group's accumulator row: word 0 = key word, then each slot's words at woff(a) (slot kinds in
// SlotKind).  DMIN / DMAX words hold dord(value) so that integer min / max orders them.
template <class Ev>
WS_DI void rowIdentity(const Ev& ev, u64* w) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.woff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: w[o] = 0; break;
      case SK_ISUM: w[o] = 0, w[o + 1] = 0; break;
      case SK_IMIN: w[o] = (u64)0x7fffffffffffffffll; break;
      case SK_IMAX: w[o] = (u64)0x8000000000000000ll; break;
      case SK_DSUM: w[o] = 0; break;
      case SK_DMIN: w[o] = (u64)dord(__longlong_as_double(0x7ff0000000000000ll)); break;
      case SK_DMAX: w[o] = (u64)dord(__longlong_as_double((i64)0xfff0000000000000ull)); break;
      default: break;
    }
  }
}
// Adds row `i` of the current 4-row group into accumulator words w (registers).
template <class Ev>
WS_DI void rowAccumulate(const Ev& ev, int i, u64* w) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.woff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: w[o] += 1; break;
      case SK_ISUM: {
        i64 v;
        if (ev.ival(a, i, v)) add128(w[o], *(i64*)&w[o + 1], v);
        break;
      }
      case SK_IMIN: {
        i64 v;
        if (ev.ival(a, i, v) && v < (i64)w[o]) w[o] = (u64)v;
        break;
      }
      case SK_IMAX: {
        i64 v;
        if (ev.ival(a, i, v) && v > (i64)w[o]) w[o] = (u64)v;
        break;
      }
      case SK_DSUM: {
        const double v = ev.dval(a, i);
        if (v == v) w[o] = (u64)__double_as_longlong(__longlong_as_double((i64)w[o]) + v);
        break;
      }
      case SK_DMIN: {
        const double v = ev.dval(a, i);
        if (v == v && dord(v) < (i64)w[o]) w[o] = (u64)dord(v);
        break;
      }
      case SK_DMAX: {
        const double v = ev.dval(a, i);
        if (v == v && dord(v) > (i64)w[o]) w[o] = (u64)dord(v);
        break;
      }
      default: break;
    }
  }
}
// w += x (both accumulator rows, same layout)
template <class Ev>
WS_DI void rowCombine(const Ev& ev, u64* w, const u64* x) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.woff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: w[o] += x[o]; break;
      case SK_ISUM: add128w(w[o], *(i64*)&w[o + 1], x[o], (i64)x[o + 1]); break;
      case SK_IMIN: case SK_DMIN: if ((i64)x[o] < (i64)w[o]) w[o] = x[o]; break;
      case SK_IMAX: case SK_DMAX: if ((i64)x[o] > (i64)w[o]) w[o] = x[o]; break;
      case SK_DSUM:
        w[o] = (u64)__double_as_longlong(__longlong_as_double((i64)w[o]) + __longlong_as_double((i64)x[o]));
        break;
      default: break;
    }
  }
}
// Atomic w += x into a row in shared or global memory (generic addressing).
template <class Ev>
WS_DI void rowAtomicCombine(const Ev& ev, u64* w, const u64* x) {
#pragma unroll
  for (int a = 0; a < Ev::NA; ++a) {
    if (a >= ev.na()) break;
    const int o = ev.woff(a);
    switch (ev.kind(a)) {
      case SK_COUNT: if (x[o]) atomicAdd(w + o, x[o]); break;
      case SK_ISUM: if (x[o] || x[o + 1]) atomicAdd128(w + o, (i64*)(w + o + 1), x[o], (i64)x[o + 1]); break;
      case SK_IMIN: case SK_DMIN: if ((i64)x[o] < (i64)*(volatile u64*)(w + o)) atomicMin((i64*)(w + o), (i64)x[o]); break;
      case SK_IMAX: case SK_DMAX: if ((i64)x[o] > (i64)*(volatile u64*)(w + o)) atomicMax((i64*)(w + o), (i64)x[o]); break;
      case SK_DSUM: {
        const double v = __longlong_as_double((i64)x[o]);
        if (v != 0.0) atomicAdd((double*)(w + o), v);
        break;
      }
      default: break;
    }
  }
}
// The accumulator row of a single input row (count 1, each argument once; NULL arguments neutral).
template <class Ev>
WS_DI void rowOfInput(const Ev& ev, int i, u64* w) {
  rowIdentity(ev, w);
  rowAccumulate(ev, i, w);
}

// Warp + block reduction of one accumulator row per thread into `out` (thread 0's view).
template <class Ev, int RW>
WS_DI void blockReduceRow(const Ev& ev, u64 (&w)[RW], u64* sred /* [kStagedThreads/32][RW] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rw = ev.rowWords();
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    u64 x[RW];
#pragma unroll
    for (int j = 0; j < RW; ++j) x[j] = j < rw ? __shfl_down_sync(0xffffffffu, w[j], off) : 0;
    rowCombine(ev, w, x);
  }
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < RW; ++j)
      if (j < rw) sred[warp * RW + j] = w[j];
  __syncthreads();
  if (warp == 0) {
    if (lane < (int)(blockDim.x >> 5)) {
#pragma unroll
      for (int j = 0; j < RW; ++j)
        if (j < rw) w[j] = sred[lane * RW + j];
    } else {
      rowIdentity(ev, w);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      u64 x[RW];
#pragma unroll
      for (int j = 0; j < RW; ++j) x[j] = j < rw ? __shfl_down_sync(0xffffffffu, w[j], off) : 0;
      rowCombine(ev, w, x);
    }
  }
  __syncthreads();
}

// After every CTA wrote its partial rows part[cta][nrows][rw]: the last CTA to finish reduces them
// into rows[nrows][rw] (word 0 of each row = its key word, left as is).  Thread t folds CTAs t,
// t + blockDim, ... in order, then a fixed-shape tree combines the threads: deterministic.
template <class Ev, int RW>
WS_DI void lastCtaReduce(const Launch& L, const Ev& ev, int nrows, u64* sred) {
  __shared__ bool amLast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) amLast = atomicAdd(L.ticket, 1u) == ctaCount(L) - 1;
  __syncthreads();
  if (!amLast) return;
  __threadfence();
  const int rw = ev.rowWords();
  for (int g = 0; g < nrows; ++g) {
    u64 w[RW];
    rowIdentity(ev, w);
    for (unsigned c = threadIdx.x; c < ctaCount(L); c += blockDim.x) {
      const u64* p = L.part + ((size_t)c * nrows + g) * rw;
      u64 x[RW];
#pragma unroll
      for (int j = 1; j < RW; ++j) x[j] = j < rw ? __ldcg(p + j) : 0;
      rowCombine(ev, w, x);
    }
    blockReduceRow(ev, w, sred);
    if (threadIdx.x == 0) {  // rows accumulate across launches (scan windows): combine into them
      u64* out = L.rows + (size_t)g * rw;
      u64 x[RW];
#pragma unroll
      for (int j = 1; j < RW; ++j) x[j] = j < rw ? out[j] : 0;
      rowCombine(ev, x, w);
#pragma unroll
      for (int j = 1; j < RW; ++j)
        if (j < rw) out[j] = x[j];
    }
  }
}

// ------------------------------------------------------------------ no GROUP BY
template <class Ev>
__device__ void aggNoKeys(const Launch& L) {
  constexpr int RW = Ev::RW, FW = Ev::FRW;
  __shared__ u64 sred[(kStagedThreads / 32) * RW];
  __shared__ u64 spill[2 * Ev::NA];
  Ev ev(L);
  for (int j = threadIdx.x; j < 2 * Ev::NA; j += blockDim.x) spill[j] = 0;
  __syncthreads();
  u64 f[FW];
  fastIdentity(ev, f);
  // register rows: a tested addition costs about what the magnitude test of the bounded form does
  // (no shared-memory ordering is at stake), so every addition is tested here
  scanRows(L, ev, [&](int i, int, i64) {
    u64 x[FW];
    fastOfInput(ev, i, x);
    fastCombine(ev, f, x, spill);
  });
  u64 w[RW];
  rowIdentity(ev, w);
  fastExpand(ev, f, w);
  __syncthreads();
  blockReduceRow(ev, w, sred);
  const int rw = ev.rowWords();
  if (threadIdx.x == 0) {
    for (int a = 0; a < ev.na(); ++a)
      if (ev.kind(a) == SK_ISUM) add128w(w[ev.woff(a)], *(i64*)&w[ev.woff(a) + 1], spill[2 * a], (i64)spill[2 * a + 1]);
    for (int j = 1; j < rw; ++j) L.part[(size_t)ctaIndex(L) * rw + j] = w[j];
  }
  lastCtaReduce<Ev, RW>(L, ev, 1, sred);
}

// ------------------------------------------------------------------ dense GROUP BY
template <class Ev>
WS_DI bool denseIndex(const Launch& L, const Ev& ev, int i, i64& g) {
  // ranges and G are below 2^26 (the dense limit), so the index arithmetic fits 32 bits
  unsigned gg = 0;
#pragma unroll
  for (int k = 0; k < Ev::NK; ++k) {
    if (k >= ev.nk()) break;
    const i64 d = ev.ikey(k, i) - L.kmin[k];
    if ((u64)d >= (u64)L.range[k]) return false;
    gg += (unsigned)d * (unsigned)L.stride[k];
  }
  g = gg;
  return gg < (unsigned)L.G;
}

// Few groups, register rows in shared memory: every thread owns G private rows laid out
// [group][word][thread] (a warp's accesses are consecutive words: no bank conflicts), so adding a row
// is one read-modify-write per word at a computed address: no atomics, no per-group predication.
// Dynamic shared memory: [stages (staged scans)][private rows G * FRW * blockDim][spill G * NA * 2].
// Each (group, word) is then reduced over the CTA's threads in a fixed order; partial rows per CTA,
// the last CTA reduces them.
template <class Ev, bool kStaged>
__device__ void aggDensePriv(const Launch& L) {
  constexpr int RW = Ev::RW, FW = Ev::FRW, T = kThreads;
  extern __shared__ __align__(16) u64 wsSmem[];
  __shared__ u64 sred[(kStagedThreads / 32) * RW];
  Ev ev(L);
  const int G = (int)L.G, tid = threadIdx.x;
  const bool owner = tid < T;  // the producer warp of a staged launch owns no rows
  const int fw = ev.fastWords();
  u64* priv = wsSmem + (size_t)(L.stages > 1 ? L.stages : 0) * (Ev::STAGE_BYTES / 8);
  u64* spill = priv + (size_t)G * fw * T;
  {
    u64 id[FW];
    fastIdentity(ev, id);
    if (owner)
      for (int g = 0; g < G; ++g)
        for (int j = 0; j < fw; ++j) priv[((size_t)g * fw + j) * T + tid] = id[j];
    for (int j = tid; j < G * 2 * Ev::NA; j += blockDim.x) spill[j] = 0;
  }
  __syncthreads();
  bool tested = false;  // this thread's sums take tested additions (sticky, see sumMagnitude)
  auto row = [&](int i, int, i64) {
    i64 gi;
    if (!denseIndex(L, ev, i, gi)) {
      L.err[0] = 1;
      return;
    }
    u64 x[FW];
    fastOfInput(ev, i, x);
    tested |= sumsNeedTests(L, sumMagnitude(ev, x));
    u64* p = priv + ((unsigned)gi * (unsigned)fw * T + tid);
    if (!tested) {  // no atomics on this path: the slots' read-modify-writes overlap
#pragma unroll
      for (int a = 0; a < Ev::NA; ++a) {
        if (a >= ev.na()) break;
        const int o = ev.fwoff(a);
        u64* q = p + (size_t)o * T;
        switch (ev.kind(a)) {
          case SK_COUNT: case SK_ISUM: *q += x[o]; break;
          case SK_IMIN: case SK_DMIN: if ((i64)x[o] < (i64)*q) *q = x[o]; break;
          case SK_IMAX: case SK_DMAX: if ((i64)x[o] > (i64)*q) *q = x[o]; break;
          case SK_DSUM: *q = (u64)__double_as_longlong(__longlong_as_double((i64)*q) + __longlong_as_double((i64)x[o])); break;
          default: break;
        }
      }
      return;
    }
    u64* sp = spill + (unsigned)gi * (2u * Ev::NA);
#pragma unroll
    for (int a = 0; a < Ev::NA; ++a) {
      if (a >= ev.na()) break;
      const int o = ev.fwoff(a);
      u64* q = p + (size_t)o * T;
      switch (ev.kind(a)) {
        case SK_COUNT: *q += x[o]; break;
        case SK_ISUM: addCarry(q, x[o], sp + 2 * a + 1); break;
        case SK_IMIN: case SK_DMIN: if ((i64)x[o] < (i64)*q) *q = x[o]; break;
        case SK_IMAX: case SK_DMAX: if ((i64)x[o] > (i64)*q) *q = x[o]; break;
        case SK_DSUM: *q = (u64)__double_as_longlong(__longlong_as_double((i64)*q) + __longlong_as_double((i64)x[o])); break;
        default: break;
      }
    }
  };
  // the direct-load entry carries no staged path (its register budget allows more resident CTAs)
  if constexpr (kStaged) scanRows(L, ev, row);
  else forEachRow(L, ev, row);
  __syncthreads();
  const int rw = ev.rowWords();
  for (int g = 0; g < G; ++g) {
    u64 f[FW];
    fastIdentity(ev, f);
    if (owner)
#pragma unroll
      for (int j = 0; j < FW; ++j)
        if (j < fw) f[j] = priv[((size_t)g * fw + j) * T + tid];
    u64 w[RW];
    rowIdentity(ev, w);
    fastExpand(ev, f, w);
    blockReduceRow(ev, w, sred);
    if (tid == 0) {
      const u64* sp = spill + (size_t)g * 2 * Ev::NA;
      for (int a = 0; a < ev.na(); ++a)
        if (ev.kind(a) == SK_ISUM) add128w(w[ev.woff(a)], *(i64*)&w[ev.woff(a) + 1], sp[2 * a], (i64)sp[2 * a + 1]);
      for (int j = 1; j < rw; ++j) L.part[((size_t)ctaIndex(L) * G + g) * rw + j] = w[j];
    }
  }
  lastCtaReduce<Ev, RW>(L, ev, G, sred);
}

// Medium G: the CTA's rows [G][rw] live in shared memory (rows' key words unused) and take shared
// atomics; at the end each non-empty group is merged into the global rows with global atomics.
template <class Ev>
__device__ void aggDenseShared(const Launch& L) {
  extern __shared__ __align__(16) u64 wsSmem[];
  Ev ev(L);
  const int rw = ev.rowWords();
  const i64 G = L.G;
  for (i64 g = threadIdx.x; g < G; g += blockDim.x) rowIdentity(ev, wsSmem + g * rw);
  __syncthreads();
  forEachRow(L, ev, [&](int i, int, i64) {
    i64 gi;
    if (!denseIndex(L, ev, i, gi)) {
      L.err[0] = 1;
      return;
    }
    u64 x[kMaxRowWords];
    rowOfInput(ev, i, x);
    rowAtomicCombine(ev, wsSmem + gi * rw, x);
  });
  __syncthreads();
  for (i64 g = threadIdx.x; g < G; g += blockDim.x) {
    const u64* s = wsSmem + g * rw;
    if (s[ev.woff(0)] == 0) continue;  // slot 0 is COUNT(*): no rows of this group in this CTA
    rowAtomicCombine(ev, L.rows + g * rw, s);
  }
}

// Large G: rows go straight to the global rows with atomics.
template <class Ev>
__device__ void aggDenseGlobal(const Launch& L) {
  Ev ev(L);
  const int rw = ev.rowWords();
  forEachRow(L, ev, [&](int i, int, i64) {
    i64 gi;
    if (!denseIndex(L, ev, i, gi)) {
      L.err[0] = 1;
      return;
    }
    u64 x[kMaxRowWords];
    rowOfInput(ev, i, x);
    rowAtomicCombine(ev, L.rows + gi * rw, x);
  });
}

// ------------------------------------------------------------------ hash GROUP BY
// Key word of a row: a single integer key is its own key word, a single double key its canonical
// bits (both exact); several keys are folded into a 64-bit hash that identifies the group, and their
// values are stored beside the table.
template <class Ev>
WS_DI u64 keyWord(const Ev& ev, int i, double* kv) {
  if (ev.nk() == 1) {
    const u64 w = ev.keyInt(0) ? (u64)ev.ikey(0, i) : (u64)dkeyBits(ev.dkey(0, i));
    kv[0] = __longlong_as_double((i64)w);
    return w;
  }
  u64 h = 0x9e3779b97f4a7c15ull;
#pragma unroll
  for (int k = 0; k < Ev::NK; ++k) {
    if (k >= ev.nk()) break;
    const u64 b = ev.keyInt(k) ? (u64)ev.ikey(k, i) : (u64)dkeyBits(ev.dkey(k, i));
    kv[k] = __longlong_as_double((i64)b);
    h = mix64(h ^ b) + (u64)k;
  }
  return h == kEmpty ? (h ^ 1) : h;
}

// Inserts accumulator row x under key word kw into the global table (linear probing, bounded).
template <class Ev>
WS_DI void globalInsert(const Launch& L, const Ev& ev, u64 kw, const double* kv, const u64* x) {
  if (*(volatile int*)(L.err + 1)) return;  // the table overflowed: the caller reruns with a bigger one
  const int rw = ev.rowWords();
  if (kw == kEmpty) {  // the EMPTY key word itself has a dedicated row after the table
    u64* row = L.table + (L.mask + 1) * rw;
    if (atomicCAS(row, 0ull, 1ull) == 0ull)
      for (int k = 0; k < ev.nk(); ++k) L.tkeys[(L.mask + 1) * ev.nk() + k] = kv[k];
    rowAtomicCombine(ev, row, x);
    return;
  }
  u64 s = mix64(kw) & L.mask;
  for (int p = 0; p < L.probeLimit; ++p) {
    u64* row = L.table + s * rw;
    u64 prev = *(volatile u64*)row;
    if (prev == kEmpty) {
      prev = atomicCAS(row, kEmpty, kw);
      if (prev == kEmpty) {
        if (ev.nk() > 1)
          for (int k = 0; k < ev.nk(); ++k) L.tkeys[s * ev.nk() + k] = kv[k];
        const u64 c = atomicAdd(L.count, 1ull) + 1;
        if (c * 10 > (L.mask + 1) * 7) L.err[1] = 1;  // fuller than 70%: the caller retries bigger
        prev = kw;
      }
    }
    if (prev == kw) {
      rowAtomicCombine(ev, row, x);
      return;
    }
    s = (s + 1) & L.mask;
  }
  L.err[1] = 1;  // no free slot within the probe limit
}

// Rows are pre-aggregated in a per-CTA shared-memory table (smemSlots rows, bounded probing), which
// absorbs hot keys.  A row that finds no slot there is appended to a per-CTA shared buffer (one
// shared atomic per warp); after each tile the whole CTA inserts the buffered rows into the global
// table together, one row per thread, so the global probes and atomics of the cold keys run with all
// lanes active instead of a few diverged lanes at a time.  (A row finding the buffer full goes to
// the global table directly.)  The shared table is merged into the global table when the CTA finishes.
// Shared memory: [S][rw] table | [S][nk] key values (multi-key) | [B][rw] buffer | [B][nk] key values.
template <class Ev>
__device__ void aggHash(const Launch& L) {
  extern __shared__ __align__(16) u64 wsSmem[];
  __shared__ int spillN, stopFlag;
  Ev ev(L);
  const int rw = ev.rowWords(), nk = ev.nk();
  const int S = L.smemSlots, B = L.spillRows;
  const bool multi = nk > 1;
  u64* tab = wsSmem;
  double* skv = (double*)(tab + (size_t)S * rw);
  u64* buf = tab + (size_t)S * rw + (multi ? (size_t)S * nk : 0);
  double* bkv = (double*)(buf + (size_t)B * rw);
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    u64* row = tab + (size_t)s * rw;
    rowIdentity(ev, row);
    row[0] = kEmpty;
  }
  if (threadIdx.x == 0) spillN = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  auto rowFn = [&](int i, int, i64) {
    double kv[Ev::NK];
    const u64 kw = keyWord(ev, i, kv);
    u64 x[kMaxRowWords];
    rowOfInput(ev, i, x);
    if (kw != kEmpty && S > 0) {
      unsigned s = (unsigned)(mix64(kw) & (u64)(S - 1));
#pragma unroll 1
      for (int p = 0; p < 8; ++p) {
        u64* row = tab + (size_t)s * rw;
        u64 prev = row[0];
        if (prev == kEmpty) {
          prev = atomicCAS(row, kEmpty, kw);
          if (prev == kEmpty) {
            if (multi)
              for (int k = 0; k < nk; ++k) skv[(size_t)s * nk + k] = kv[k];
            prev = kw;
          }
        }
        if (prev == kw) {
          rowAtomicCombine(ev, row, x);
          return;
        }
        s = (s + 1) & (S - 1);
      }
    }
    // bound for the global table: reserve a buffer entry (one shared atomic per warp)
    const unsigned m = __activemask();
    const int leader = __ffs(m) - 1, rank = __popc(m & ((1u << lane) - 1));
    int base = 0;
    if (lane == leader) base = atomicAdd(&spillN, __popc(m));
    base = __shfl_sync(m, base, leader);
    const int at = base + rank;
    if (at < B) {
      u64* e = buf + (size_t)at * rw;
      for (int w = 1; w < rw; ++w) e[w] = x[w];
      e[0] = kw;
      if (multi)
        for (int k = 0; k < nk; ++k) bkv[(size_t)at * nk + k] = kv[k];
    } else {
      globalInsert(L, ev, kw, kv, x);
    }
  };
  // Inserts the buffered rows; returns true (in every thread) once the global table has overflowed:
  // the run's result is discarded then (the caller reruns with a bigger table), so the CTA stops.
  // Barriers: the count and the flag are read between the first two, so no thread changes them (the
  // next tile's appends, the next flush's flag) before every thread has read them: the decisions
  // below are CTA-uniform.
  auto flush = [&]() -> bool {
    if (threadIdx.x == 0) stopFlag = *(volatile int*)(L.err + 1);
    __syncthreads();
    const int n = min(spillN, B);
    const bool stop = stopFlag != 0;
    __syncthreads();
    if (n == 0 || stop) return stop;
    if (threadIdx.x == 0) spillN = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const u64* e = buf + (size_t)j * rw;
      double kv[WS_MAX_KEYS];
      if (multi)
        for (int k = 0; k < nk; ++k) kv[k] = bkv[(size_t)j * nk + k];
      else
        kv[0] = __longlong_as_double((i64)e[0]);
      globalInsert(L, ev, e[0], kv, e);
    }
    __syncthreads();  // the buffer is refilled by the next tile
    return false;
  };
  forEachRowTiles(L, ev, rowFn, flush);
  if (flush()) return;  // overflowed: the shared table is not merged either
  __syncthreads();
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    const u64* row = tab + (size_t)s * rw;
    if (row[0] == kEmpty) continue;
    double kv[WS_MAX_KEYS];
    if (multi)
      for (int k = 0; k < nk; ++k) kv[k] = skv[(size_t)s * nk + k];
    else
      kv[0] = __longlong_as_double((i64)row[0]);
    globalInsert(L, ev, row[0], kv, row);
  }
}

// ------------------------------------------------------------------ selection
// Pass 1: selected rows per tile.  Pass 2 (after an exclusive scan of the tile counts): each warp
// ranks its rows with ballot / popc and writes ascending global row indices.
template <class Ev>
__device__ void selectCount(const Launch& L) {
  __shared__ int wcount[kThreads / 32];
  Ev ev(L);
  forEachOwnedTile(L, ev, [&](i64 t, int, i64 r0, i64 n, const uint32_t* del) {
    int c = 0;
    if (r0 < n) {
      const int nv = n - r0 >= 4 ? 4 : (int)(n - r0);
      ev.load(r0, ev.fastOk && nv == 4, nv);
      unsigned live = (1u << nv) - 1;
      if (del) live &= ~(__ldg(del + (r0 >> 5)) >> (r0 & 31)) & 0xfu;
#pragma unroll
      for (int i = 0; i < 4; ++i) c += ((live >> i) & 1u) && ev.where(i);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) wcount[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int w = 0; w < kThreads / 32; ++w) s += wcount[w];
      L.tileCount[t] = s;
    }
    __syncthreads();
    return false;
  });
  ev.finish();
}

template <class Ev>
__device__ void selectWrite(const Launch& L) {
  __shared__ int woff[kThreads / 32];
  Ev ev(L);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  forEachOwnedTile(L, ev, [&](i64 t, int b, i64 r0, i64 n, const uint32_t* del) {
    unsigned sel = 0;
    if (r0 < n) {
      const int nv = n - r0 >= 4 ? 4 : (int)(n - r0);
      ev.load(r0, ev.fastOk && nv == 4, nv);
      unsigned live = (1u << nv) - 1;
      if (del) live &= ~(__ldg(del + (r0 >> 5)) >> (r0 & 31)) & 0xfu;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (((live >> i) & 1u) && ev.where(i)) sel |= 1u << i;
    }
    // rank = selected rows of lower lanes (ballot per row position) + own earlier rows
    const unsigned lower = (1u << lane) - 1;
    int before = 0, total = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const unsigned m = __ballot_sync(0xffffffffu, (sel >> i) & 1u);
      before += __popc(m & lower);
      total += __popc(m);
    }
    if (lane == 0) woff[warp] = total;
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; ++w) base += woff[w];
    const i64 out0 = L.tileCount[t] + base + before;
    const i64 g0 = __ldg(L.rowStart + b) + r0;
    int k = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if ((sel >> i) & 1u) L.outIdx[out0 + k++] = (int32_t)(g0 + i);
    __syncthreads();
    return false;
  });
  ev.finish();
}

}  // namespace ws

// Kernel entry points (extern "C" names so generated modules can be looked up by name).  The Launch
// descriptor is a __grid_constant__ parameter: the evaluator keeps a reference to it without forcing a
// per-thread copy.
#define WS_K_ENTRY_B(PREFIX, NAME, BODY, THREADS, MINB)                                                      \
  extern "C" __global__ void __launch_bounds__(THREADS, MINB) PREFIX##_##NAME(const __grid_constant__ ws::Launch L) { \
    BODY(L);                                                                                                 \
  }
#define WS_K_ENTRY(PREFIX, NAME, BODY) WS_K_ENTRY_B(PREFIX, NAME, BODY, ws::kStagedThreads, 1)
// The same body serving several queries in one launch: each CTA finds its query (binary search of the
// CTA ranges) and runs the body on a shared-memory copy of that query's descriptor with its CTA range.
#define WS_K_MULTI_B(PREFIX, NAME, BODY, THREADS, MINB)                                                       \
  extern "C" __global__ void __launch_bounds__(THREADS, MINB) PREFIX##_multi_##NAME(const __grid_constant__ ws::MultiLaunch M) { \
    __shared__ __align__(16) ws::Launch Lq;                                                                 \
    int lo = 0, hi = M.nq - 1;                                                                               \
    while (lo < hi) {                                                                                        \
      const int mid = (lo + hi + 1) >> 1;                                                                    \
      if (M.ctaStart[mid] <= (int)blockIdx.x) lo = mid;                                                      \
      else hi = mid - 1;                                                                                     \
    }                                                                                                        \
    const unsigned long long* src = (const unsigned long long*)(M.q + lo);                                  \
    for (int w = threadIdx.x; w < (int)(sizeof(ws::Launch) / 8); w += blockDim.x) ((unsigned long long*)&Lq)[w] = src[w]; \
    __syncthreads();                                                                                         \
    if (threadIdx.x == 0) Lq.ctaBase = M.ctaStart[lo], Lq.ctaGrid = M.ctaStart[lo + 1] - M.ctaStart[lo];    \
    __syncthreads();                                                                                         \
    BODY(Lq);                                                                                                \
  }
#define WS_K_MULTI_NOKEYS(EV, PREFIX) WS_K_MULTI_B(PREFIX, nokeys, ws::aggNoKeys<EV>, ws::kStagedThreads, 1)
#define WS_K_MULTI_DENSE_PRIV(EV, PREFIX) \
  WS_K_MULTI_B(PREFIX, dense_priv, (ws::aggDensePriv<EV, false>), ws::kThreads, EV::PRIV_MIN_BLOCKS)
// The hash scan launches kThreads.  For generated plans EV::HASH_MULTI_MIN_BLOCKS = 3 resident CTAs
// (the shared table allows them) bound the registers: reading the launch descriptor from shared
// memory took the kernel from 72 to 82 registers, two CTAs per SM and 20 % more time than the
// single-query scan; bounded it needs 80, without spills.
#define WS_K_MULTI_HASH(EV, PREFIX) \
  WS_K_MULTI_B(PREFIX, hash, ws::aggHash<EV>, ws::kThreads, EV::HASH_MULTI_MIN_BLOCKS)
#define WS_K_NOKEYS(EV, PREFIX) WS_K_ENTRY(PREFIX, nokeys, ws::aggNoKeys<EV>)
#define WS_K_DENSE_SHARED(EV, PREFIX) WS_K_ENTRY(PREFIX, dense_shared, ws::aggDenseShared<EV>)
#define WS_K_DENSE_GLOBAL(EV, PREFIX) WS_K_ENTRY(PREFIX, dense_global, ws::aggDenseGlobal<EV>)
// The direct-load private-row kernel asks for EV::PRIV_MIN_BLOCKS resident CTAs of kThreads (a
// register budget); the staged one keeps the producer warp.
#define WS_K_DENSE_PRIV(EV, PREFIX)                                                                      \
  WS_K_ENTRY_B(PREFIX, dense_priv, (ws::aggDensePriv<EV, false>), ws::kThreads, EV::PRIV_MIN_BLOCKS)     \
  WS_K_ENTRY(PREFIX, dense_priv_staged, (ws::aggDensePriv<EV, true>))
#define WS_K_HASH(EV, PREFIX) WS_K_ENTRY(PREFIX, hash, ws::aggHash<EV>)
#define WS_K_SELECT_COUNT(EV, PREFIX) WS_K_ENTRY(PREFIX, select_count, ws::selectCount<EV>)
#define WS_K_SELECT_WRITE(EV, PREFIX) WS_K_ENTRY(PREFIX, select_write, ws::selectWrite<EV>)
#define WS_DEFINE_SCAN_KERNELS(EV, PREFIX) \
  WS_K_NOKEYS(EV, PREFIX)                  \
  WS_K_DENSE_SHARED(EV, PREFIX)            \
  WS_K_DENSE_GLOBAL(EV, PREFIX)            \
  WS_K_DENSE_PRIV(EV, PREFIX)              \
  WS_K_HASH(EV, PREFIX)                    \
  WS_K_SELECT_COUNT(EV, PREFIX)            \
  WS_K_SELECT_WRITE(EV, PREFIX)
