// Filter + aggregate without GROUP BY that allocates no memory.
//
// Some callers cannot allocate device memory: code that runs where the allocator is off limits, for
// example inside a host callback, under a memory budget enforced by another component, or a caller
// whose only memory is what it was handed.  ws_agg_nokeys_noalloc gives them the no-key aggregation of
// ws_agg_* using a fixed scratch area that lives in this library's module: a file-scope __device__
// array of WS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the process exits.
// The batch descriptor, the per-CTA partial rows, the result row and the control words all live there;
// the caller passes the inputs (column views) and a host array for the result.
//
// All calls share the one array, which keeps the last call's contents: each call clears and
// re-initialises what must start at a known value (control words, result row) before its launch.
// Calls whose work overlaps on the GPU (other threads, other streams) race on the array; callers must
// serialise them.  The first call on a device looks up the array's device address (once per device,
// with that device current); make that first call before any stream capture begins.
#include <cstring>

#include "ws_internal.h"

namespace ws {
namespace {

// Scratch: [control 256 B][result row 2 KiB][descriptor 1 MiB][partial rows rest]
static __device__ __align__(256) unsigned char gNoAllocScratch[WS_NOALLOC_SCRATCH_BYTES];
constexpr size_t kCtlOff = 0, kRowOff = 256, kDescOff = 256 + 2048, kDescBytes = 1 << 20;
constexpr size_t kPartOff = kDescOff + kDescBytes, kPartBytes = WS_NOALLOC_SCRATCH_BYTES - kPartOff;

std::mutex gMu;
unsigned char* gScratch[64] = {};  // device address of the array, per device ordinal

unsigned char* scratchOnDevice() {
  int dev = 0;
  WS_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error("device ordinal out of range", WS_ERR_ARG);
  std::lock_guard<std::mutex> g(gMu);
  if (!gScratch[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, gNoAllocScratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw Error(std::string("no-allocation scratch unavailable: ") + cudaGetErrorString(e), WS_ERR_INTERNAL);
    }
    gScratch[dev] = (unsigned char*)p;
  }
  return gScratch[dev];
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" int ws_agg_nokeys_noalloc(const ws_expr_env* env, int ncols, const ws_agg_plan* plan,
                                     const ws_jit_program* jit, int nb, const int64_t* bn, const uint32_t* const* bdel,
                                     const ws_col_view* bcols, int64_t* exact) {
  return guardedCall([&] {
    if (!env || !plan || !exact || (nb > 0 && (!bn || !bcols))) throw Error("null argument", WS_ERR_ARG);
    if (plan->nkeys != 0) throw Error("ws_agg_nokeys_noalloc aggregates without GROUP BY keys only", WS_ERR_ARG);
    if (ncols < 0 || ncols > WS_MAX_COLS || nb < 0) throw Error("bad column or batch count", WS_ERR_ARG);
    const SlotLayout lay = layoutOf(*plan);
    const bool useJit = jit && jit->state.load() == 1 && jit->kernels.fn[K_NOKEYS] &&
                        [&] {
                          for (int b = 0; b < nb; ++b)
                            for (int c = 0; c < ncols; ++c)
                              if (bcols[(int64_t)b * ncols + c].enc && !env->cols[c].enc) return false;
                          return true;
                        }();
    if (!useJit && plan->naggs > WS_INTERP_AGGS)
      throw Error("this aggregation needs a compiled plan (more than 16 aggregates)", WS_ERR_PLAN);
    // descriptor layout (as the allocating path uploads it)
    size_t off = 0;
    auto take = [&](size_t bytes) {
      const size_t o = align16(off);
      off = o + bytes;
      return o;
    };
    const size_t oCols = take((size_t)nb * ncols * sizeof(ws_col_view)), oN = take(8 * (size_t)nb),
                 oDel = take(8 * (size_t)nb), oTile = take(8 * ((size_t)nb + 1)), oRow = take(8 * ((size_t)nb + 1));
    size_t oProg = 0, oKinds = 0, oWoff = 0, oFwoff = 0, oNull = 0, oKeyInt = 0;
    if (!useJit) {
      oProg = take(sizeof(TProgs));
      oKinds = take(WS_MAX_AGGS);
      oWoff = take(4 * WS_MAX_AGGS);
      oFwoff = take(4 * WS_MAX_AGGS);
      oNull = take(WS_MAX_AGGS);
      oKeyInt = take(WS_MAX_KEYS);
    }
    if (off > kDescBytes)
      throw Error("ws_agg_nokeys_noalloc: " + std::to_string(nb) + " batches x " + std::to_string(ncols) +
                      " columns need " + std::to_string(off) + " descriptor bytes; the fixed scratch holds " +
                      std::to_string(kDescBytes),
                  WS_ERR_SIZE);
    std::vector<uint8_t> st(std::max<size_t>(off, 16), 0);
    if (nb) memcpy(st.data() + oCols, bcols, (size_t)nb * ncols * sizeof(ws_col_view));
    int64_t* n = (int64_t*)(st.data() + oN);
    const uint32_t** del = (const uint32_t**)(st.data() + oDel);
    int64_t *ts = (int64_t*)(st.data() + oTile), *rs = (int64_t*)(st.data() + oRow);
    ts[0] = rs[0] = 0;
    for (int b = 0; b < nb; ++b) {
      n[b] = std::max<int64_t>(bn[b], 0);
      del[b] = bdel ? bdel[b] : nullptr;
      ts[b + 1] = ts[b] + (n[b] + kTile - 1) / kTile;
      rs[b + 1] = rs[b] + n[b];
    }
    const int64_t ntiles = ts[nb];
    if (!useJit) {
      TProgs progs;
      buildTProgs(*env, ncols, *plan, plan->hasWhere, progs);
      memcpy(st.data() + oProg, &progs, sizeof progs);
      memcpy(st.data() + oKinds, lay.kind, WS_MAX_AGGS);
      memcpy(st.data() + oWoff, lay.woff, 4 * WS_MAX_AGGS);
      memcpy(st.data() + oFwoff, lay.fwoff, 4 * WS_MAX_AGGS);
      memcpy(st.data() + oNull, plan->aggNull, WS_MAX_AGGS);
      memcpy(st.data() + oKeyInt, plan->keyInt, WS_MAX_KEYS);
    }
    ensureInit();
    unsigned char* s = scratchOnDevice();
    const KernelSet& ks = useJit ? jit->kernels : interpKernels();
    CUfunction f = ks.fn[K_NOKEYS];
    unsigned grid = persistentGrid(f, 0, std::max<int64_t>(ntiles, 1));
    const unsigned maxGrid = (unsigned)(kPartBytes / (8 * (size_t)lay.rw));
    if (grid > maxGrid) grid = maxGrid;
    // the result row starts at the aggregates' identities; control words at zero
    std::vector<u64> row(lay.rw, 0);
    for (int a = 0; a < lay.na; ++a) {
      const int o = lay.woff[a];
      double inf = __builtin_inf(), ninf = -__builtin_inf();
      long long bi, bn2;
      memcpy(&bi, &inf, 8);
      memcpy(&bn2, &ninf, 8);
      switch (lay.kind[a]) {
        case SK_IMIN: row[o] = (u64)0x7fffffffffffffffll; break;
        case SK_IMAX: row[o] = (u64)0x8000000000000000ll; break;
        case SK_DMIN: row[o] = (u64)(bi >= 0 ? bi : (bi ^ 0x7fffffffffffffffll)); break;
        case SK_DMAX: row[o] = (u64)(bn2 >= 0 ? bn2 : (bn2 ^ 0x7fffffffffffffffll)); break;
        default: break;
      }
    }
    WS_CK(cudaMemsetAsync(s + kCtlOff, 0, 256, stream()));
    WS_CK(cudaMemcpyAsync(s + kRowOff, row.data(), 8 * (size_t)lay.rw, cudaMemcpyHostToDevice, stream()));
    if (ntiles > 0) {
      WS_CK(cudaMemcpyAsync(s + kDescOff, st.data(), off, cudaMemcpyHostToDevice, stream()));
      Launch L;
      memset(&L, 0, sizeof L);
      unsigned char* d = s + kDescOff;
      L.cols = (const ws_col_view*)(d + oCols);
      L.n = (const i64*)(d + oN);
      L.del = (const uint32_t* const*)(d + oDel);
      L.tileStart = (const i64*)(d + oTile);
      L.rowStart = (const i64*)(d + oRow);
      L.nb = nb;
      L.ncols = ncols;
      L.ntiles = ntiles;
      L.env = envK(*env);
      if (!useJit) {
        L.progs = (const TProgs*)(d + oProg);
        L.kinds = d + oKinds;
        L.woff = (const int*)(d + oWoff);
        L.fwoff = (const int*)(d + oFwoff);
        L.aggNull = d + oNull;
        L.keyInt = d + oKeyInt;
      }
      L.nkeys = 0;
      L.naggs = plan->naggs;
      L.rowWords = lay.rw;
      L.fastWords = lay.frw;
      L.rows = (u64*)(s + kRowOff);
      L.part = (u64*)(s + kPartOff);
      L.err = (int*)(s + kCtlOff);
      L.ticket = (unsigned*)(s + kCtlOff + 24);
      L.stages = 0;
      launchScan(f, grid, 0, L);
    }
    std::vector<u64> out(lay.rw);
    int err[3];
    WS_CK(cudaMemcpyAsync(out.data(), s + kRowOff, 8 * (size_t)lay.rw, cudaMemcpyDeviceToHost, stream()));
    WS_CK(cudaMemcpyAsync(err, s + kCtlOff, sizeof err, cudaMemcpyDeviceToHost, stream()));
    WS_CK(cudaStreamSynchronize(stream()));
    if (err[2]) throw Error("a staged tile copy did not complete in time", WS_ERR_INTERNAL);
    for (int a = 0; a < plan->naggs; ++a) {  // exact words, the layout of ws_agg_fetch's `exact`
      const int src = lay.kind[a] == SK_NONE ? lay.partner[a] : a;
      const int o = lay.woff[src];
      long long w0 = (long long)out[o], w1 = 0;
      if (lay.kind[src] == SK_ISUM) w1 = (long long)out[o + 1];
      else if (lay.kind[src] == SK_DMIN || lay.kind[src] == SK_DMAX) w0 = w0 >= 0 ? w0 : (w0 ^ 0x7fffffffffffffffll);
      exact[2 * a] = w0;
      exact[2 * a + 1] = w1;
    }
  });
}
