// Tiered column storage and column-level UPDATE: the VRAM budget of segment columns, host columns
// pinned and mapped for zero-copy reads when the budget is full, and new device copies of a column
// with some rows changed (reference: src/gpu.cu:82-155, :229-369; declarations src/gpu.h:19-47).
//
// Device copies made here are plain cudaMalloc allocations (persistent, outside the stream-ordered
// pool) counted against one process-wide budget; the engine releases them with ws_release_column /
// ws_vram_release.  The UPDATE kernels write one new copy of the column: the old copy stays valid for
// readers until the engine swaps the pointer.
#include <climits>
#include <cmath>
#include <cstring>

#include "ws_internal.h"

namespace ws {
namespace {

std::atomic<int64_t> gVramUsed{0};
std::atomic<int64_t> gVramLimit{INT64_MAX};

bool fits(size_t bytes) { return gVramUsed.load() + (int64_t)bytes <= gVramLimit.load(); }

// A counted device allocation, or nullptr when the device has no room (the error is cleared).
void* countedAlloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  gVramUsed += (int64_t)bytes;
  return p;
}
void countedFree(void* p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  gVramUsed -= (int64_t)bytes;
}

int gridFor(int64_t n) {
  int64_t g = (n + 255) / 256;
  const int64_t cap = (int64_t)smCount() * 8;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}
#define WS_GRID_STRIDE(j, n) \
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < (n); j += (int64_t)gridDim.x * blockDim.x)

// col[rows[i]] = vals[i] (4- or 8-byte elements)
__global__ void kPatch(uint8_t* col, int w, const int32_t* rows, const uint8_t* vals, int64_t m) {
  WS_GRID_STRIDE(i, m) {
    if (w == 8) ((u64*)col)[rows[i]] = ((const u64*)vals)[i];
    else ((uint32_t*)col)[rows[i]] = ((const uint32_t*)vals)[i];
  }
}

// Result of kUpdate: min / max of the written non-NULL values as order-preserving keys, flags.
struct UpdateOut {
  u64 mnKey, mxKey;
  int bad, sawNull;
};
// double -> unsigned key with the same order (negative values: all bits flipped; others: sign set)
__device__ __forceinline__ u64 orderKey(double v) {
  const u64 b = (u64)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double fromOrderKey(u64 k) {
  const u64 b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  memcpy(&v, &b, 8);
  return v;
}

// One warp-level pass over the listed rows: each thread folds its rows' new values into a local
// min / max and flags, then one atomic per warp publishes them.
__global__ void kUpdate(uint8_t* dst, const uint8_t* src, int w, int f64, const int32_t* rows, int64_t m,
                        const __grid_constant__ ws_update u, UpdateOut* out) {
  double mn = INFINITY, mx = -INFINITY;
  int bad = 0, sawNull = 0;
  WS_GRID_STRIDE(i, m) {
    const int32_t r = rows[i];
    if (f64) {
      double v = u.d0;
      if (u.kind) {
        v = ((const double*)src)[r];
        if (v != v) {
          bad |= u.not_null;
          sawNull = 1;
        } else {
          v += u.add_d;
        }
      }
      ((double*)dst)[r] = v;
      if (v == v) mn = fmin(mn, v), mx = fmax(mx, v);
      continue;
    }
    i64 v = u.i0;
    if (u.kind) {
      v = w == 8 ? ((const i64*)src)[r] : (i64)((const int*)src)[r];
      if (v == u.nul) {
        bad |= u.not_null;
        sawNull = 1;
      } else if (u.kind == 2) {
        unsigned of = 0;
        v = iaddf(v, u.add, of);  // checked: an overflow is a value out of range
        bad |= (int)of;
      }
    }
    if (v != u.nul && (v < u.lo || v > u.hi)) bad = 1;
    if (w == 8) ((i64*)dst)[r] = v;
    else ((int*)dst)[r] = (int)v;
    if (v != u.nul) mn = fmin(mn, (double)v), mx = fmax(mx, (double)v);
  }
  // warp reduction of the flags and of the order keys, one lane publishes
  const unsigned full = 0xffffffffu;
  bad = __any_sync(full, bad);
  sawNull = __any_sync(full, sawNull);
  u64 kmn = mn <= mx ? orderKey(mn) : ~0ull, kmx = mn <= mx ? orderKey(mx) : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    const u64 a = __shfl_xor_sync(full, kmn, o), b = __shfl_xor_sync(full, kmx, o);
    kmn = a < kmn ? a : kmn;
    kmx = b > kmx ? b : kmx;
  }
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicOr(&out->bad, 1);
    if (sawNull) atomicOr(&out->sawNull, 1);
    if (kmn != ~0ull) atomicMin((unsigned long long*)&out->mnKey, kmn);
    if (kmx != 0ull) atomicMax((unsigned long long*)&out->mxKey, kmx);
  }
}

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

int ws_set_vram_limit(int64_t bytes) {
  return guardedCall([&] {
    if (bytes < 0) throw Error("ws_set_vram_limit: negative limit", WS_ERR_ARG);
    gVramLimit = bytes;
  });
}
int64_t ws_vram_used(void) { return gVramUsed.load(); }
int64_t ws_vram_limit(void) { return gVramLimit.load(); }
int64_t ws_vram_free(void) {
  size_t fr = 0, total = 0;
  if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (int64_t)fr;
}
double ws_vram_fill(void) {
  const int64_t lim = gVramLimit.load();
  if (lim != INT64_MAX) return lim > 0 ? (double)gVramUsed.load() / (double)lim : 1.0;
  size_t fr = 0, total = 1;
  if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return 1.0 - (double)fr / (double)total;
}

int ws_place_column(void* host, size_t bytes, int host_only, void** out, int* mapped) {
  return guardedCall([&] {
    ensureInit();
    *out = nullptr;
    *mapped = 0;
    if (!bytes) return;
    if (!host_only && fits(bytes)) {
      void* p = countedAlloc(bytes);
      if (!p) {  // memory the pool holds may be returned to the device
        WS_CK(cudaDeviceSynchronize());
        WS_CK(cudaMemPoolTrimTo([] {
          cudaMemPool_t pool;
          int dev = 0;
          cudaGetDevice(&dev);
          cudaDeviceGetDefaultMemPool(&pool, dev);
          return pool;
        }(), 0));
        p = countedAlloc(bytes);
      }
      if (p) {
        const cudaError_t e = cudaMemcpy(p, host, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
          countedFree(p, bytes);
          ck(e, "placeColumn: copy to the device");
        }
        *out = p;
        return;
      }
    }
    WS_CK(cudaHostRegister(host, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable));
    void* d = nullptr;
    const cudaError_t e = cudaHostGetDevicePointer(&d, host, 0);
    if (e != cudaSuccess) {
      cudaHostUnregister(host);
      ck(e, "placeColumn: mapping host memory");
    }
    *out = d;
    *mapped = 1;
  });
}

int ws_release_column(void* dev, void* host, size_t bytes, int mapped) {
  return guardedCall([&] {
    if (!dev) return;
    if (mapped) WS_CK(cudaHostUnregister(host));
    else countedFree(dev, bytes);
  });
}

int ws_vram_acquire(const void* host, size_t bytes, void** out) {
  return guardedCall([&] {
    ensureInit();
    *out = nullptr;
    if (!bytes || !fits(bytes)) return;
    void* p = countedAlloc(bytes);
    if (!p) return;
    const cudaError_t e = cudaMemcpy(p, host, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      countedFree(p, bytes);
      ck(e, "vramAcquire: copy to the device");
    }
    *out = p;
  });
}

int ws_vram_release(void* dev, size_t bytes) {
  return guardedCall([&] { countedFree(dev, bytes); });
}

int ws_host_map(void* host, size_t bytes, void** out) {
  return guardedCall([&] {
    ensureInit();
    *out = nullptr;
    if (cudaHostRegister(host, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, host, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaHostUnregister(host);
      return;
    }
    *out = d;
  });
}

int ws_host_unmap(void* host) {
  return guardedCall([&] {
    if (cudaHostUnregister(host) != cudaSuccess) cudaGetLastError();
  });
}

int ws_patch_column(const void* old_dev, size_t bytes, int width, const int32_t* rows, const void* vals, int64_t m,
                    void** out) {
  return guardedCall([&] {
    ensureInit();
    *out = nullptr;
    if (m < 0) throw Error("ws_patch_column: negative row count", WS_ERR_ARG);
    if ((width != 4 && width != 8) || !fits(bytes)) return;
    void* p = countedAlloc(bytes);
    if (!p) return;
    try {
      WS_CK(cudaMemcpyAsync(p, old_dev, bytes, cudaMemcpyDeviceToDevice, stream()));
      if (m > 0) {
        const size_t rb = ((size_t)m * 4 + 15) / 16 * 16, vb = (size_t)m * width;
        uint8_t* st = pinnedStage(rb + vb);
        memcpy(st, rows, (size_t)m * 4);
        memcpy(st + rb, vals, vb);
        DBuf<uint8_t> d((int64_t)(rb + vb));
        WS_CK(cudaMemcpyAsync(d.p, st, rb + vb, cudaMemcpyHostToDevice, stream()));
        stageCopied();
        kPatch<<<gridFor(m), 256, 0, stream()>>>((uint8_t*)p, width, (const int32_t*)d.p, d.p + rb, m);
        WS_CK(cudaGetLastError());
        countLaunch();
      }
      WS_CK(cudaStreamSynchronize(stream()));
    } catch (...) {
      cudaStreamSynchronize(stream());
      countedFree(p, bytes);
      throw;
    }
    *out = p;
  });
}

int ws_update_column(const void* old_dev, const void* src, int64_t n, int w, int f64, const int32_t* rows, int64_t m,
                     ws_update* u, void** out) {
  return guardedCall([&] {
    ensureInit();
    *out = nullptr;
    u->bad = 0;
    if (n < 0 || m < 0) throw Error("ws_update_column: negative size", WS_ERR_ARG);
    const size_t bytes = (size_t)n * (size_t)w;
    if ((w != 4 && w != 8) || !fits(bytes)) return;
    void* p = countedAlloc(bytes);
    if (!p) return;
    UpdateOut res{~0ull, 0ull, 0, 0};
    try {
      WS_CK(cudaMemcpyAsync(p, old_dev, bytes, cudaMemcpyDeviceToDevice, stream()));
      if (m > 0) {
        const size_t rb = ((size_t)m * 4 + 15) / 16 * 16;
        uint8_t* st = pinnedStage(rb + sizeof(UpdateOut));
        memcpy(st, rows, (size_t)m * 4);
        memcpy(st + rb, &res, sizeof res);
        DBuf<uint8_t> d((int64_t)(rb + sizeof(UpdateOut)));
        WS_CK(cudaMemcpyAsync(d.p, st, rb + sizeof(UpdateOut), cudaMemcpyHostToDevice, stream()));
        stageCopied();
        UpdateOut* dout = (UpdateOut*)(d.p + rb);
        kUpdate<<<gridFor(m), 256, 0, stream()>>>((uint8_t*)p, (const uint8_t*)src, w, f64, (const int32_t*)d.p, m, *u,
                                                  dout);
        WS_CK(cudaGetLastError());
        countLaunch();
        d2hSync(&res, dout, sizeof res);
      }
      WS_CK(cudaStreamSynchronize(stream()));
    } catch (...) {
      cudaStreamSynchronize(stream());
      countedFree(p, bytes);
      throw;
    }
    u->bad = res.bad != 0;
    u->saw_null = res.sawNull != 0;
    u->mn = res.mnKey == ~0ull ? INFINITY : fromOrderKey(res.mnKey);
    u->mx = res.mxKey == 0ull ? -INFINITY : fromOrderKey(res.mxKey);
    if (u->bad) {
      countedFree(p, bytes);
      return;
    }
    *out = p;
  });
}

}  // extern "C"
