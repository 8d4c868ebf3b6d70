// Device helpers shared by the ahead-of-time library kernels (nvcc) and the per-query kernels compiled
// at run time (NVRTC, sm_100a).  No host headers: this file is embedded verbatim into every generated
// query source.
//
// Contents: SQL value semantics (NULL = NaN in double-typed expressions, sentinels in integer storage,
// three-valued logic, checked int64 arithmetic), segment column decoding, 128-bit vector loads,
// exact 128-bit integer accumulation, and the launch descriptor every scan kernel receives.
#pragma once
#include "ws_types.h"

#define WS_DI __device__ __forceinline__

namespace ws {

typedef unsigned long long u64;
typedef long long i64;

// ------------------------------------------------------------------ values
WS_DI double nanv() { return __longlong_as_double(0x7ff8000000000000ll); }
WS_DI bool isnul(double v) { return v != v; }
WS_DI bool truthy(double v) { return v == v && v != 0.0; }
// canonical group-key bits of a double key: -0.0 groups with +0.0, every NaN with the canonical NaN
WS_DI i64 dkeyBits(double d) {
  d = d + 0.0;
  return d != d ? 0x7ff8000000000000ll : __double_as_longlong(d);
}

// three-valued comparison / logic over doubles (src/devtypes.h:248-270)
WS_DI double cmp3(int op, double a, double b) {
  if (a != a || b != b) return nanv();
  bool r;
  switch (op) {
    case 0: r = a == b; break;
    case 1: r = a != b; break;
    case 2: r = a < b; break;
    case 3: r = a <= b; break;
    case 4: r = a > b; break;
    default: r = a >= b; break;
  }
  return r ? 1.0 : 0.0;
}
WS_DI double and3(double a, double b) {
  if ((a == a && a == 0.0) || (b == b && b == 0.0)) return 0.0;
  if (a != a || b != b) return nanv();
  return 1.0;
}
WS_DI double or3(double a, double b) {
  if ((a == a && a != 0.0) || (b == b && b != 0.0)) return 1.0;
  if (a != a || b != b) return nanv();
  return 0.0;
}
WS_DI double not3(double a) { return a != a ? a : (a == 0.0 ? 1.0 : 0.0); }
WS_DI double coalesce2(double a, double b) { return a != a ? b : a; }
WS_DI double nullif2(double a, double b) { return a == b ? nanv() : a; }
WS_DI double divz(double a, double b) { return b == 0.0 ? nanv() : a / b; }
WS_DI double nullIfI32(i64 v) { return v == (i64)WS_NULL_I32 ? nanv() : (double)v; }
WS_DI double nullIfI64(i64 v) { return v == (i64)WS_NULL_I64 ? nanv() : (double)v; }
WS_DI double decOf(i64 v, double p10) { return v == (i64)WS_NULL_I64 ? nanv() : (double)v / p10; }

// checked int64 arithmetic: wraps like two's complement and raises the query's overflow flag
WS_DI i64 iaddc(i64 a, i64 b, int* f) {
  const i64 r = (i64)((u64)a + (u64)b);
  if (((a ^ r) & (b ^ r)) < 0 && f) *f = 1;
  return r;
}
WS_DI i64 isubc(i64 a, i64 b, int* f) {
  const i64 r = (i64)((u64)a - (u64)b);
  if (((a ^ b) & (a ^ r)) < 0 && f) *f = 1;
  return r;
}
WS_DI i64 imulc(i64 a, i64 b, int* f) {
  if (a == (i64)(int)a && b == (i64)(int)b) return (i64)(int)a * (i64)(int)b;  // 32 x 32 bits: exact
  const i64 r = (i64)((u64)a * (u64)b);
  if (__mul64hi(a, b) != (r >> 63) && f) *f = 1;
  return r;
}
// The same checked operations with the overflow accumulated into a register (bit 0 of `of`; no
// branch and no store per operation): generated evaluators OR it into their flag once per thread.
WS_DI i64 iaddf(i64 a, i64 b, unsigned& of) {
  const i64 r = (i64)((u64)a + (u64)b);
  of |= (unsigned)((u64)((a ^ r) & (b ^ r)) >> 63);
  return r;
}
WS_DI i64 isubf(i64 a, i64 b, unsigned& of) {
  const i64 r = (i64)((u64)a - (u64)b);
  of |= (unsigned)((u64)((a ^ b) & (a ^ r)) >> 63);
  return r;
}
// 32 x 32-bit product of the operands' low words, exact when both operands fit in int32; `wide` collects
// the operands that do not (the caller then recomputes with imulf).  Branch-free.
WS_DI i64 imul32w(i64 a, i64 b, unsigned& wide) {
  wide |= ((unsigned)((u64)a >> 32) ^ (unsigned)((int)a >> 31)) | ((unsigned)((u64)b >> 32) ^ (unsigned)((int)b >> 31));
  return (i64)(int)a * (i64)(int)b;
}
WS_DI i64 imulf(i64 a, i64 b, unsigned& of) {
  if (a == (i64)(int)a && b == (i64)(int)b) return (i64)(int)a * (i64)(int)b;  // 32 x 32 bits: exact
  const i64 r = (i64)((u64)a * (u64)b);
  of |= (unsigned)(__mul64hi(a, b) != (r >> 63));
  return r;
}

WS_DI i64 insetI(const uint32_t* bits, int size, i64 c) {
  return (c >= 0 && c < size) ? (i64)((__ldg(bits + (c >> 5)) >> (c & 31)) & 1u) : 0ll;
}
WS_DI double insetD(const uint32_t* bits, int size, double x) {
  if (x != x) return x;
  return (double)insetI(bits, size, (i64)x);
}
WS_DI double insortedD(const double* a, int n, double x) {
  if (x != x) return x;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < n && __ldg(a + lo) == x ? 1.0 : 0.0;
}
WS_DI double dictmapD(const double* map, int size, double x) {
  if (x != x) return x;
  const i64 c = (i64)x;
  return (c >= 0 && c < size) ? __ldg(map + c) : nanv();
}
WS_DI double vecD(bool dot, const float* v, i64 row, const double* q, int dim) {
  const float* x = v + row * (i64)dim;
  if (x[0] != x[0]) return nanv();
  float acc = 0.f;
  for (int i = 0; i < dim; ++i) {
    if (dot) {
      acc += x[i] * (float)q[i];
    } else {
      const float d = x[i] - (float)q[i];
      acc += d * d;
    }
  }
  return dot ? (double)acc : sqrt((double)acc);
}

// ---- calendar: Howard Hinnant's public-domain civil-date algorithms (days_from_civil /
// civil_from_days), proleptic Gregorian, day 0 = 1970-01-01.
WS_DI i64 daysFromCivil(i64 y, unsigned m, unsigned d) {
  y -= m <= 2;
  const i64 era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = (unsigned)(y - era * 400);
  const unsigned doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + (i64)doe - 719468;
}
WS_DI void civilFromDays(i64 z, i64& y, unsigned& m, unsigned& d) {
  z += 719468;
  const i64 era = (z >= 0 ? z : z - 146096) / 146097;
  const unsigned doe = (unsigned)(z - era * 146097);
  const unsigned yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  y = (i64)yoe + era * 400;
  const unsigned doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const unsigned mp = (5 * doy + 2) / 153;
  d = doy - (153 * mp + 2) / 5 + 1;
  m = mp < 10 ? mp + 3 : mp - 9;
  y += (m <= 2);
}
WS_DI i64 yearOf(i64 days) {
  i64 y;
  unsigned m, d;
  civilFromDays(days, y, m, d);
  return y;
}
WS_DI i64 floorDiv(i64 a, i64 b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
WS_DI i64 addMonthsDays(i64 days, i64 n) {
  i64 y;
  unsigned m, d;
  civilFromDays(days, y, m, d);
  const i64 months = y * 12 + (m - 1) + n;
  y = months >= 0 ? months / 12 : (months - 11) / 12;
  m = (unsigned)(months - y * 12) + 1;
  const unsigned mdays = m == 2 ? 28u : (m == 4 || m == 6 || m == 9 || m == 11) ? 30u : 31u;
  const bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
  const unsigned lim = mdays + (m == 2 && leap);
  return daysFromCivil(y, m, d < lim ? d : lim);
}

// scalar functions by id (src/devtypes.h:324-427); math goes to the CUDA math library
static __device__ __noinline__ double call1(int fn, double x) {
  if (x != x) return x;
  const i64 usd = 86400000000ll;
  i64 y;
  unsigned m, d;
  const i64 xi = (i64)x;
  switch (fn) {
    case WS_FN_ABS: return x < 0 ? -x : x;
    case WS_FN_CEIL: return ceil(x);
    case WS_FN_FLOOR: return floor(x);
    case WS_FN_ROUND: return round(x);
    case WS_FN_SQRT: return x < 0 ? nanv() : sqrt(x);
    case WS_FN_EXP: return exp(x);
    case WS_FN_LN: return x <= 0 ? nanv() : log(x);
    case WS_FN_LOG10: return x <= 0 ? nanv() : log10(x);
    case WS_FN_LOG2: return x <= 0 ? nanv() : log2(x);
    case WS_FN_SIN: return sin(x);
    case WS_FN_COS: return cos(x);
    case WS_FN_TAN: return tan(x);
    case WS_FN_ASIN: return asin(x);
    case WS_FN_ACOS: return acos(x);
    case WS_FN_ATAN: return atan(x);
    case WS_FN_DEGREES: return x * (180.0 / 3.14159265358979323846);
    case WS_FN_RADIANS: return x * (3.14159265358979323846 / 180.0);
    case WS_FN_SIGN: return x > 0 ? 1.0 : x < 0 ? -1.0 : 0.0;
    case WS_FN_MONTH: civilFromDays(xi, y, m, d); return m;
    case WS_FN_DAY: civilFromDays(xi, y, m, d); return d;
    case WS_FN_DAYOFWEEK: return (double)((xi + 4) - floorDiv(xi + 4, 7) * 7 + 1);
    case WS_FN_WEEKDAY: return (double)((xi + 3) - floorDiv(xi + 3, 7) * 7);
    case WS_FN_DAYOFYEAR: civilFromDays(xi, y, m, d); return (double)(xi - daysFromCivil(y, 1, 1) + 1);
    case WS_FN_QUARTER: civilFromDays(xi, y, m, d); return (double)((m - 1) / 3 + 1);
    case WS_FN_WEEK:
    case WS_FN_YEARWEEK: {
      civilFromDays(xi, y, m, d);
      const i64 jan1 = daysFromCivil(y, 1, 1);
      const i64 dow = (jan1 + 4) - floorDiv(jan1 + 4, 7) * 7;
      const i64 firstSun = jan1 + (7 - dow) % 7;
      const double wk = xi < firstSun ? 0.0 : (double)((xi - firstSun) / 7 + 1);
      return fn == WS_FN_WEEK ? wk : (double)(y * 100) + wk;
    }
    case WS_FN_LAST_DAY: civilFromDays(xi, y, m, d); return (double)(addMonthsDays(daysFromCivil(y, m, 1), 1) - 1);
    case WS_FN_TO_DAYS: return x + 719528;
    case WS_FN_FROM_DAYS: return x - 719528;
    case WS_FN_DT_DATE: return (double)floorDiv(xi, usd);
    case WS_FN_DT_HOUR: return (double)((xi - floorDiv(xi, usd) * usd) / 3600000000ll);
    case WS_FN_DT_MINUTE: return (double)(((xi - floorDiv(xi, usd) * usd) / 60000000ll) % 60);
    case WS_FN_DT_SECOND: return (double)(((xi - floorDiv(xi, usd) * usd) / 1000000ll) % 60);
    case WS_FN_DT_MICRO: return (double)(xi - floorDiv(xi, 1000000ll) * 1000000ll);
    case WS_FN_DATE_TO_DT: return x * (double)usd;
    case WS_FN_DT_UNIX: return floor(x / 1e6);
    case WS_FN_UNIX_DT: return x * 1e6;
    case WS_FN_DT_YEAR: civilFromDays(floorDiv(xi, usd), y, m, d); return (double)y;
    case WS_FN_DT_MONTH: civilFromDays(floorDiv(xi, usd), y, m, d); return m;
    case WS_FN_DT_DAY: civilFromDays(floorDiv(xi, usd), y, m, d); return d;
  }
  return nanv();
}
static __device__ __noinline__ double call2(int fn, double a, double b) {
  if (a != a || b != b) return nanv();
  const i64 usd = 86400000000ll;
  switch (fn) {
    case WS_FN_LEAST: return a < b ? a : b;
    case WS_FN_GREATEST: return a > b ? a : b;
    case WS_FN_ROUND2: { const double p = pow(10.0, b); return round(a * p) / p; }
    case WS_FN_TRUNCATE2: { const double p = pow(10.0, b); return trunc(a * p) / p; }
    case WS_FN_POW: return pow(a, b);
    case WS_FN_ATAN2: return atan2(a, b);
    case WS_FN_LOG_B: return (a <= 0 || b <= 0) ? nanv() : log(b) / log(a);
    case WS_FN_IDIV: return b == 0 ? nanv() : trunc(a / b);
    case WS_FN_ADD_MONTHS: return (double)addMonthsDays((i64)a, (i64)b);
    case WS_FN_DT_ADD_MONTHS: {
      const i64 us = (i64)a, days = floorDiv(us, usd);
      return (double)(addMonthsDays(days, (i64)b) * usd + (us - days * usd));
    }
    case WS_FN_DATE_TRUNC_MONTH: {
      i64 y;
      unsigned m, d;
      civilFromDays((i64)a, y, m, d);
      return (double)daysFromCivil(y, b > 0 ? 1 : m, 1);
    }
  }
  return nanv();
}
// YEAR of a double-typed date expression (src/jit.cu:231-236)
WS_DI double yearD(double x) { return call1(WS_FN_DT_YEAR, call1(WS_FN_DATE_TO_DT, x)); }

// ------------------------------------------------------------------ exact accumulation
// 128-bit integer as (lo, hi) words; add of a sign-extended int64
WS_DI void add128(u64& lo, i64& hi, i64 v) {
  asm("add.cc.u64 %0, %0, %2;\n\taddc.s64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(v), "l"(v >> 63));
}
WS_DI void add128w(u64& lo, i64& hi, u64 vlo, i64 vhi) {
  asm("add.cc.u64 %0, %0, %2;\n\taddc.s64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(vlo), "l"(vhi));
}
// order-preserving map of doubles to signed int64 (for atomic MIN / MAX of doubles)
WS_DI i64 dord(double d) {
  const i64 b = __double_as_longlong(d);
  return b >= 0 ? b : (b ^ 0x7fffffffffffffffll);
}
WS_DI double dunord(i64 k) { return __longlong_as_double(k >= 0 ? k : (k ^ 0x7fffffffffffffffll)); }

// shared-memory / global atomics on a 128-bit (lo, hi) pair: exact for any interleaving
WS_DI void atomicAdd128(u64* lo, i64* hi, u64 vlo, i64 vhi) {
  const u64 old = atomicAdd(lo, vlo);
  const i64 carry = (old + vlo < old) ? 1 : 0;
  const i64 h = vhi + carry;
  if (h) atomicAdd((u64*)hi, (u64)h);
}

// ------------------------------------------------------------------ loads
// streaming 128-bit loads of read-only segment data (no L1 allocation: each byte is used once)
WS_DI int4 ldg4(const void* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
WS_DI int2 ldg2(const void* p) {
  int2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.s32 {%0,%1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  return v;
}
WS_DI unsigned ldg1(const void* p) {
  unsigned v;
  asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Four consecutive rows of a column.  `fast`: the group is full and its address is aligned to
// min(16, 4 * width) bytes (checked per batch); otherwise per-row loads of the first nv rows.
WS_DI void load4i32(int (&o)[4], const int* p, bool fast, int nv) {
  if (fast) {
    const int4 v = ldg4(p);
    o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = i < nv ? __ldg(p + i) : 0;
  }
}
WS_DI void load4i64(i64 (&o)[4], const i64* p, bool fast, int nv) {
  if (fast) {
    const int4 a = ldg4(p), b = ldg4(p + 2);
    o[0] = (i64)(((u64)(unsigned)a.y << 32) | (unsigned)a.x);
    o[1] = (i64)(((u64)(unsigned)a.w << 32) | (unsigned)a.z);
    o[2] = (i64)(((u64)(unsigned)b.y << 32) | (unsigned)b.x);
    o[3] = (i64)(((u64)(unsigned)b.w << 32) | (unsigned)b.z);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = i < nv ? __ldg(p + i) : 0;
  }
}
WS_DI void load4f64(double (&o)[4], const double* p, bool fast, int nv) {
  i64 t[4];
  load4i64(t, (const i64*)p, fast, nv);
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = __longlong_as_double(t[i]);
}
// Encoded integer column (enc 1/2/3: uint8/16/32 offsets from base; the all-ones code is NULL).
// `d` points at the codes of row 0 (header skipped, range-scan offset applied).
WS_DI void load4enc(i64 (&o)[4], const unsigned char* d, int enc, i64 base, i64 nul, bool fast, int nv) {
  unsigned c[4];
  if (enc == 1) {
    if (fast) {
      const unsigned v = ldg1(d);
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = (v >> (8 * i)) & 0xffu;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = i < nv ? (unsigned)__ldg(d + i) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = c[i] == 0xffu ? nul : base + (i64)c[i];
  } else if (enc == 2) {
    const unsigned short* s = (const unsigned short*)d;
    if (fast) {
      const int2 v = ldg2(s);
      c[0] = (unsigned)v.x & 0xffffu, c[1] = (unsigned)v.x >> 16, c[2] = (unsigned)v.y & 0xffffu, c[3] = (unsigned)v.y >> 16;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = i < nv ? (unsigned)__ldg(s + i) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = c[i] == 0xffffu ? nul : base + (i64)c[i];
  } else {
    const unsigned* s = (const unsigned*)d;
    if (fast) {
      const int4 v = ldg4(s);
      c[0] = (unsigned)v.x, c[1] = (unsigned)v.y, c[2] = (unsigned)v.z, c[3] = (unsigned)v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = i < nv ? __ldg(s + i) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = c[i] == 0xffffffffu ? nul : base + (i64)c[i];
  }
}
// Encoded double column: enc 4 = 256-entry dictionary + uint8 codes; enc 5/6 = decimal-valued doubles
// as uint16/uint32 offsets from base divided by p10 (the all-ones code is NULL).
WS_DI void load4encD(double (&o)[4], const unsigned char* d, const double* dict, int enc, i64 base, double p10,
                     bool fast, int nv) {
  if (enc == 4) {
    unsigned c[4];
    if (fast) {
      const unsigned v = ldg1(d);
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = (v >> (8 * i)) & 0xffu;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) c[i] = i < nv ? (unsigned)__ldg(d + i) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = __ldg(dict + c[i]);
    return;
  }
  i64 t[4];
  load4enc(t, d, enc == 5 ? 2 : 3, base, (i64)WS_NULL_I64, fast, nv);
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = t[i] == (i64)WS_NULL_I64 ? nanv() : (double)t[i] / p10;
}

// The same 4-row loads from a shared-memory stage (generic addressing; the stage holds whole tiles, so
// every group is full and aligned).
WS_DI void stage4i32(int (&o)[4], const unsigned char* p) {
  const int4 v = *(const int4*)p;
  o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w;
}
WS_DI void stage4i64(i64 (&o)[4], const unsigned char* p) {
  const longlong2 a = *(const longlong2*)p, b = *(const longlong2*)(p + 16);
  o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
}
WS_DI void stage4f64(double (&o)[4], const unsigned char* p) {
  const double2 a = *(const double2*)p, b = *(const double2*)(p + 16);
  o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
}
WS_DI void stage4enc(i64 (&o)[4], const unsigned char* p, int enc, i64 base, i64 nul) {
  unsigned c[4], top;
  if (enc == 1) {
    const unsigned v = *(const unsigned*)p;
    for (int i = 0; i < 4; ++i) c[i] = (v >> (8 * i)) & 0xffu;
    top = 0xffu;
  } else if (enc == 2) {
    const uint2 v = *(const uint2*)p;
    c[0] = v.x & 0xffffu, c[1] = v.x >> 16, c[2] = v.y & 0xffffu, c[3] = v.y >> 16;
    top = 0xffffu;
  } else {
    const uint4 v = *(const uint4*)p;
    c[0] = v.x, c[1] = v.y, c[2] = v.z, c[3] = v.w;
    top = 0xffffffffu;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = c[i] == top ? nul : base + (i64)c[i];
}
WS_DI void stage4encD(double (&o)[4], const unsigned char* p, const double* dict, int enc, i64 base, double p10) {
  if (enc == 4) {
    const unsigned v = *(const unsigned*)p;
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = __ldg(dict + ((v >> (8 * i)) & 0xffu));
    return;
  }
  i64 t[4];
  stage4enc(t, p, enc == 5 ? 2 : 3, base, (i64)WS_NULL_I64);
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = t[i] == (i64)WS_NULL_I64 ? nanv() : (double)t[i] / p10;
}

// ---- bulk asynchronous copies (TMA engine, non-tensor form) into shared memory, completed on an
// mbarrier.  No cluster multicast: every copy reads this GPU's own memory into this CTA.
WS_DI unsigned smemAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
WS_DI void mbarInit(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
WS_DI void fenceMbarInit() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
WS_DI void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
WS_DI void mbarArriveTx(unsigned bar, unsigned tx) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx) : "memory");
}
WS_DI void mbarArrive(unsigned bar) { asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory"); }
WS_DI bool mbarTest(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity; gives up after about 2^log2Limit SM cycles (32: ~2 s) and
// returns false.
WS_DI bool mbarWait(unsigned bar, unsigned parity, int log2Limit = 32) {
  if (mbarTest(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbarTest(bar, parity)) {
    if (clock64() - t0 > (1ll << log2Limit)) return false;
    __nanosleep(32);
  }
  return true;
}
// global -> shared bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned)
WS_DI void bulkG2S(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// ---- bit-packed (enc 7) and run-length (enc 8) integer segments (formats of this library; the
// engine's own FOR / dictionary / decimal encodings are enc 1-6).
//   enc 7: header [int64 base][int32 bits b (1..32)][int32 0], then the codes packed LSB-first in
//          little-endian 32-bit words (code of stored row i = bits [i*b, i*b + b)), then 16 pad bytes;
//          value = base + code, the all-ones code is NULL.
//   enc 8: header [int64 runs][int64 0], then int32 ends[runs] (exclusive end row of each run,
//          ascending; padded to 8 bytes), then int64 vals[runs] (the stored value, NULL sentinels
//          included).
// Row r of a view with range-scan offset `off` is stored row r + off.  Decoded out of line (the
// reference decodes its encoded columns out of line too) so the inline FOR loads stay small.
WS_DI unsigned bitpackCode(const unsigned* w, i64 i, int b) {
  const u64 bit = (u64)i * (unsigned)b;
  const u64 word = bit >> 5;
  const unsigned sh = (unsigned)(bit & 31);
  const u64 two = (u64)__ldg(w + word) | ((u64)__ldg(w + word + 1) << 32);
  return (unsigned)(two >> sh) & (b == 32 ? 0xffffffffu : ((1u << b) - 1u));
}
WS_DI i64 rleRun(const int* ends, i64 runs, i64 i) {  // first run whose end is above stored row i
  i64 lo = 0, hi = runs;
  while (lo < hi) {
    const i64 mid = (lo + hi) >> 1;
    if ((i64)__ldg(ends + mid) <= i) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
// Rows r0 .. r0+nv-1 of an enc 7 / enc 8 integer view.
static __device__ __noinline__ void load4encView(i64* o, const ws_col_view* vp, i64 r0, i64 nul, int nv) {
  const ws_col_view v = *vp;
  const unsigned char* p = (const unsigned char*)v.p;
  const i64 i0 = r0 + v.off;
  if (v.enc == 7) {
    const i64 base = *(const i64*)p;
    const int b = *(const int*)(p + 8);
    const unsigned* w = (const unsigned*)(p + WS_ENC_HEADER);
    const unsigned nulc = b == 32 ? 0xffffffffu : ((1u << b) - 1u);
    for (int k = 0; k < 4; ++k) {
      if (k >= nv) {
        o[k] = 0;
        continue;
      }
      const unsigned c = bitpackCode(w, i0 + k, b);
      o[k] = c == nulc ? nul : base + (i64)c;
    }
    return;
  }
  const i64 runs = *(const i64*)p;
  const int* ends = (const int*)(p + WS_ENC_HEADER);
  const i64* vals = (const i64*)(p + WS_ENC_HEADER + ((runs * 4 + 7) & ~7ll));
  i64 run = rleRun(ends, runs, i0);
  for (int k = 0; k < 4; ++k) {
    if (k >= nv) {
      o[k] = 0;
      continue;
    }
    while (run < runs && (i64)__ldg(ends + run) <= i0 + k) ++run;
    o[k] = run < runs ? __ldg(vals + run) : nul;
  }
}

// Resolved view of one column of the current batch: where row 0's data starts and how it is encoded.
struct ColRef {
  const unsigned char* d;  // data of row 0 (raw: the view pointer; encoded: header skipped + off applied)
  const double* dict;      // enc 4 dictionary
  i64 base;                // enc 1/2/3/5/6 base
  double p10;              // enc 5/6 divisor
  int enc;
  int width;               // bytes per stored row
};
WS_DI ColRef resolveCol(const ws_col_view& v) {
  ColRef c;
  c.enc = v.enc;
  const unsigned char* p = (const unsigned char*)v.p;
  if (!v.enc) {
    c.d = p;
    c.dict = nullptr;
    c.base = 0;
    c.p10 = 1.0;
    c.width = (v.t == 0 || v.t == 3) ? 4 : 8;
    return c;
  }
  c.width = (v.enc == 1 || v.enc == 4) ? 1 : (v.enc == 2 || v.enc == 5) ? 2 : v.enc >= 7 ? 0 : 4;  // 7 / 8: packed
  c.base = p ? *(const i64*)p : 0;
  c.p10 = p ? *(const double*)(p + 8) : 1.0;
  c.dict = (const double*)(p + WS_ENC_HEADER);
  c.d = p + WS_ENC_HEADER + (v.enc == 4 ? 256 * 8 : 0) + (i64)v.off * c.width;
  return c;
}
WS_DI bool aligned4(const ColRef& c) {
  if (c.width == 0) return true;  // enc 7 / 8 decode element-wise
  const unsigned a = c.width * 4 < 16 ? c.width * 4 : 16;
  return ((unsigned long long)c.d & (a - 1)) == 0;
}

// ------------------------------------------------------------------ launch descriptor
// Query constants by value (kernel parameter space: broadcast to every thread at no memory cost).
struct EnvK {
  double consts[WS_MAX_CONSTS];
  const uint32_t* sets[WS_MAX_SETS];
  int setSize[WS_MAX_SETS];
  const double* maps[WS_MAX_SETS];
  int mapSize[WS_MAX_SETS];
  int* ovf;
};

// Typed bytecode for the on-device interpreter (built on the host from the engine's bytecode).
struct TInstr {
  uint8_t op;     // ws_op
  uint8_t rInt;   // result type: 1 int64, 0 double
  uint8_t aInt;   // operand types (first / second / third)
  uint8_t bInt;
  uint8_t cInt;
  uint8_t pad;
  uint16_t arg;
};
struct TProgs {
  int where[2];            // start, len in `code` (len 0: no program)
  int keys[WS_MAX_KEYS][2];
  int aggs[WS_MAX_AGGS][2];
  TInstr code[1024];
};

// Slot kinds of the accumulator layout (fixed when the plan is prepared on the host).
enum SlotKind : uint8_t {
  SK_NONE = 0,   // derived slot (high half of a split BIGINT SUM): no accumulation
  SK_COUNT,      // rows
  SK_ISUM,       // exact int128 SUM (2 words)
  SK_IMIN, SK_IMAX,
  SK_DSUM, SK_DMIN, SK_DMAX
};
WS_DI int slotWords(int k) { return k == SK_NONE ? 0 : k == SK_ISUM ? 2 : 1; }

struct Launch {
  // batches
  const ws_col_view* cols;    // [nb * ncols]
  const i64* n;               // [nb]
  const uint32_t* const* del; // [nb]
  const i64* tileStart;       // [nb + 1]: first tile of each batch
  const i64* rowStart;        // [nb + 1]: first global row of each batch
  int nb, ncols;
  i64 ntiles;
  EnvK env;
  const TProgs* progs;        // interpreter only
  const uint8_t* kinds;       // interpreter only: SlotKind per slot
  const int* woff;            // interpreter only: word offset per slot
  const uint8_t* aggNull;     // interpreter only
  const uint8_t* keyInt;      // interpreter only
  const int* fwoff;           // interpreter only: word offset per slot in register rows
  int nkeys, naggs, rowWords; // interpreter only (JIT: compile-time)
  int fastWords;              // interpreter only: words of a register row
  int stages;                 // shared-memory stages of staged scans (0: loads straight from global memory)
  int sumShift;               // integer SUM words need no overflow test while (argument magnitude >> sumShift)
                              // is 0 (set at launch from the rows a thread adds; -1: always test)
  int waitLog2;               // staged scans: a wait for a tile stage gives up after 2^waitLog2 SM cycles
  // A launch serving several queries gives each its own range of CTAs: this query's first CTA and its
  // CTA count (0: the whole grid).  Bodies use ctaIndex / ctaCount, never blockIdx / gridDim.
  int ctaBase, ctaGrid;
  // aggregation outputs
  u64* part;                  // per-CTA partial rows
  u64* rows;                  // result rows
  unsigned* ticket;           // last-CTA-done counter (zeroed before launch)
  int* err;                   // error flags: [0] dense key out of range, [1] hash table overflow,
                              // [2] a staged tile did not arrive in time
  // dense GROUP BY
  i64 G;
  i64 kmin[WS_MAX_KEYS], range[WS_MAX_KEYS], stride[WS_MAX_KEYS];
  // hash GROUP BY
  u64* table;                 // [cap + 1] rows of rowWords words (word 0: key word); the extra row holds the EMPTY key
  double* tkeys;              // [cap * nkeys] key values (multi-key / double keys)
  u64 mask;                   // cap - 1
  u64* count;                 // occupied rows
  int smemSlots;              // per-CTA shared table slots (power of 2)
  int spillRows;              // per-CTA shared buffer of rows bound for the global table (hash GROUP BY)
  int probeLimit;             // global probe limit before reporting overflow
  // selection
  i64* tileCount;             // [ntiles] selected rows per tile (count pass) / exclusive offsets (write pass)
  int32_t* outIdx;
};

WS_DI unsigned ctaIndex(const Launch& L) { return blockIdx.x - (unsigned)L.ctaBase; }
WS_DI unsigned ctaCount(const Launch& L) { return L.ctaGrid ? (unsigned)L.ctaGrid : gridDim.x; }

// One launch of a scan kernel over several queries of the same compiled plan: query q's launch
// descriptor q[q] and CTAs [ctaStart[q], ctaStart[q + 1]).
struct MultiLaunch {
  const Launch* q;
  const int* ctaStart;  // [nq + 1]
  int nq;
};

}  // namespace ws
