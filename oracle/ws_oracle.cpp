#include <climits>
// CPU oracle of the Warpstore hot-path operators — TEST INFRASTRUCTURE ONLY (see ws_oracle.h).
//
// The expression semantics follow the reference's typed code generator (src/jit.cu:113-273), which is
// the path the engine runs with codegen on: integer-typed nodes are evaluated in checked int64
// arithmetic, every other node in doubles with SQL three-valued logic (NULL = NaN,
// src/devtypes.h:248-304).  Expressions are evaluated a block of rows at a time (each node yields an
// array of values), which keeps the oracle fast enough to serve as the timed CPU baseline.
#include "ws_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

typedef __int128 i128;
constexpr int kBlock = 1024;
constexpr int64_t kLLMax = INT64_MAX, kLLMin = INT64_MIN;

double nanv() {
  uint64_t u = 0x7ff8000000000000ull;
  double d;
  memcpy(&d, &u, 8);
  return d;
}
inline int64_t dbits(double d) {
  int64_t v;
  memcpy(&v, &d, 8);
  return v;
}
inline double bitsd(int64_t v) {
  double d;
  memcpy(&d, &v, 8);
  return d;
}
inline bool isnan_(double v) { return v != v; }
inline bool truthy(double v) { return v == v && v != 0; }

// ---------------------------------------------------------------- column decoding
// src/devtypes.h:91-158 (encIntB, encDbl, colInt, colDbl) and :217-245 (loadCol).
int64_t colInt(const ws_col_view& c, int64_t r) {
  if (c.enc == 7) {  // bit-packed: [int64 base][int32 bits][int32 0], codes LSB-first in 32-bit words
    const unsigned char* p = (const unsigned char*)c.p;
    int64_t base;
    int32_t b;
    memcpy(&base, p, 8);
    memcpy(&b, p + 8, 4);
    const uint64_t bit = (uint64_t)(r + c.off) * (uint64_t)b;
    uint64_t two = 0;
    memcpy(&two, p + WS_ENC_HEADER + (bit >> 5) * 4, 8);
    const uint64_t mask = b == 32 ? 0xffffffffull : ((1ull << b) - 1);
    const uint64_t code = (two >> (bit & 31)) & mask;
    const int64_t nul = (c.t == 0 || c.t == 3) ? (int64_t)WS_NULL_I32 : WS_NULL_I64;
    return code == mask ? nul : base + (int64_t)code;
  }
  if (c.enc == 8) {  // run-length: [int64 runs][int64 0], int32 ends[runs] (padded to 8 B), int64 vals[runs]
    const unsigned char* p = (const unsigned char*)c.p;
    int64_t runs;
    memcpy(&runs, p, 8);
    const int32_t* ends = (const int32_t*)(p + WS_ENC_HEADER);
    const int64_t* vals = (const int64_t*)(p + WS_ENC_HEADER + ((runs * 4 + 7) & ~7ll));
    const int64_t i = r + c.off;
    const int64_t k = std::upper_bound(ends, ends + runs, (int32_t)i) - ends;
    return k < runs ? vals[k] : ((c.t == 0 || c.t == 3) ? (int64_t)WS_NULL_I32 : WS_NULL_I64);
  }
  if (c.enc) {
    const unsigned char* d = (const unsigned char*)c.p + WS_ENC_HEADER;
    const int64_t i = r + c.off;
    int64_t base;
    memcpy(&base, c.p, 8);
    const int64_t nul = (c.t == 0 || c.t == 3) ? (int64_t)WS_NULL_I32 : WS_NULL_I64;
    if (c.enc == 1) { const unsigned v = d[i]; return v == 0xFFu ? nul : base + v; }
    if (c.enc == 2) { uint16_t v; memcpy(&v, d + 2 * i, 2); return v == 0xFFFFu ? nul : base + v; }
    uint32_t v;
    memcpy(&v, d + 4 * i, 4);
    return v == 0xFFFFFFFFu ? nul : base + (int64_t)v;
  }
  if (c.t == 0 || c.t == 3) return ((const int32_t*)c.p)[r];
  return ((const int64_t*)c.p)[r];
}
double colDbl(const ws_col_view& c, int64_t r) {
  if (!c.enc) return ((const double*)c.p)[r];
  const unsigned char* d = (const unsigned char*)c.p + WS_ENC_HEADER;
  if (c.enc == 4) {
    const unsigned code = d[256 * 8 + r + c.off];
    double v;
    memcpy(&v, d + 8 * code, 8);
    return v;
  }
  int64_t base;
  double p10;
  memcpy(&base, c.p, 8);
  memcpy(&p10, (const unsigned char*)c.p + 8, 8);
  const int64_t i = r + c.off;
  if (c.enc == 5) {
    uint16_t v;
    memcpy(&v, d + 2 * i, 2);
    return v == 0xFFFFu ? nanv() : (double)(base + v) / p10;
  }
  uint32_t v;
  memcpy(&v, d + 4 * i, 4);
  return v == 0xFFFFFFFFu ? nanv() : (double)(base + (int64_t)v) / p10;
}
double pow10i(int s) {
  double p = 1;
  for (int i = 0; i < s; ++i) p *= 10;
  return p;
}

// ---------------------------------------------------------------- scalar semantics
// Civil-date conversions: Howard Hinnant's public-domain "chrono-compatible low-level date
// algorithms" (days_from_civil / civil_from_days), as the reference uses (src/devtypes.h:40-61).
int64_t daysFromCivil(int64_t y, unsigned m, unsigned d) {
  y -= m <= 2;
  const int64_t era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = (unsigned)(y - era * 400);
  const unsigned doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + (int64_t)doe - 719468;
}
void civilFromDays(int64_t z, int64_t& y, unsigned& m, unsigned& d) {
  z += 719468;
  const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  const unsigned doe = (unsigned)(z - era * 146097);
  const unsigned yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  y = (int64_t)yoe + era * 400;
  const unsigned doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const unsigned mp = (5 * doy + 2) / 153;
  d = doy - (153 * mp + 2) / 5 + 1;
  m = mp < 10 ? mp + 3 : mp - 9;
  y += (m <= 2);
}
int64_t floorDiv(int64_t a, int64_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
constexpr int64_t kUsPerDay = 86400000000ll;
int64_t addMonthsDays(int64_t days, int64_t n) {
  int64_t y;
  unsigned m, d;
  civilFromDays(days, y, m, d);
  const int64_t months = y * 12 + (m - 1) + n;
  y = months >= 0 ? months / 12 : (months - 11) / 12;
  m = (unsigned)(months - y * 12) + 1;
  static const unsigned mdays[] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  const bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
  const unsigned lim = mdays[m - 1] + (m == 2 && leap);
  return daysFromCivil(y, m, d < lim ? d : lim);
}
// One-argument scalar functions (src/devtypes.h:324-394).
double call1(int fn, double x) {
  if (isnan_(x)) return x;
  int64_t y;
  unsigned m, d;
  const int64_t xi = (int64_t)x;
  switch (fn) {
    case WS_FN_ABS: return x < 0 ? -x : x;
    case WS_FN_CEIL: return std::ceil(x);
    case WS_FN_FLOOR: return std::floor(x);
    case WS_FN_ROUND: return std::round(x);
    case WS_FN_SQRT: return x < 0 ? nanv() : std::sqrt(x);
    case WS_FN_EXP: return std::exp(x);
    case WS_FN_LN: return x <= 0 ? nanv() : std::log(x);
    case WS_FN_LOG10: return x <= 0 ? nanv() : std::log10(x);
    case WS_FN_LOG2: return x <= 0 ? nanv() : std::log2(x);
    case WS_FN_SIN: return std::sin(x);
    case WS_FN_COS: return std::cos(x);
    case WS_FN_TAN: return std::tan(x);
    case WS_FN_ASIN: return std::asin(x);
    case WS_FN_ACOS: return std::acos(x);
    case WS_FN_ATAN: return std::atan(x);
    case WS_FN_DEGREES: return x * (180.0 / M_PI);
    case WS_FN_RADIANS: return x * (M_PI / 180.0);
    case WS_FN_SIGN: return x > 0 ? 1.0 : x < 0 ? -1.0 : 0.0;
    case WS_FN_MONTH: civilFromDays(xi, y, m, d); return m;
    case WS_FN_DAY: civilFromDays(xi, y, m, d); return d;
    case WS_FN_DAYOFWEEK: return (double)((xi + 4) - floorDiv(xi + 4, 7) * 7 + 1);  // 1 = Sunday
    case WS_FN_WEEKDAY: return (double)((xi + 3) - floorDiv(xi + 3, 7) * 7);        // 0 = Monday
    case WS_FN_DAYOFYEAR: civilFromDays(xi, y, m, d); return (double)(xi - daysFromCivil(y, 1, 1) + 1);
    case WS_FN_QUARTER: civilFromDays(xi, y, m, d); return (double)((m - 1) / 3 + 1);
    case WS_FN_WEEK: {
      civilFromDays(xi, y, m, d);
      const int64_t jan1 = daysFromCivil(y, 1, 1);
      const int64_t dow = (jan1 + 4) - floorDiv(jan1 + 4, 7) * 7;  // 0 = Sunday
      const int64_t firstSun = jan1 + (7 - dow) % 7;
      return xi < firstSun ? 0.0 : (double)((xi - firstSun) / 7 + 1);
    }
    case WS_FN_YEARWEEK: civilFromDays(xi, y, m, d); return (double)(y * 100) + call1(WS_FN_WEEK, x);
    case WS_FN_LAST_DAY: civilFromDays(xi, y, m, d); return (double)(addMonthsDays(daysFromCivil(y, m, 1), 1) - 1);
    case WS_FN_TO_DAYS: return x + 719528;
    case WS_FN_FROM_DAYS: return x - 719528;
    case WS_FN_DT_DATE: return (double)floorDiv(xi, kUsPerDay);
    case WS_FN_DT_HOUR: return (double)((xi - floorDiv(xi, kUsPerDay) * kUsPerDay) / 3600000000ll);
    case WS_FN_DT_MINUTE: return (double)(((xi - floorDiv(xi, kUsPerDay) * kUsPerDay) / 60000000ll) % 60);
    case WS_FN_DT_SECOND: return (double)(((xi - floorDiv(xi, kUsPerDay) * kUsPerDay) / 1000000ll) % 60);
    case WS_FN_DT_MICRO: return (double)(xi - floorDiv(xi, 1000000ll) * 1000000ll);
    case WS_FN_DATE_TO_DT: return x * (double)kUsPerDay;
    case WS_FN_DT_UNIX: return std::floor(x / 1e6);
    case WS_FN_UNIX_DT: return x * 1e6;
    case WS_FN_DT_YEAR: civilFromDays(floorDiv(xi, kUsPerDay), y, m, d); return (double)y;
    case WS_FN_DT_MONTH: civilFromDays(floorDiv(xi, kUsPerDay), y, m, d); return m;
    case WS_FN_DT_DAY: civilFromDays(floorDiv(xi, kUsPerDay), y, m, d); return d;
  }
  return nanv();
}
// Two-argument scalar functions (src/devtypes.h:396-427).
double call2(int fn, double a, double b) {
  if (isnan_(a) || isnan_(b)) return nanv();
  switch (fn) {
    case WS_FN_LEAST: return a < b ? a : b;
    case WS_FN_GREATEST: return a > b ? a : b;
    case WS_FN_ROUND2: { const double p = std::pow(10.0, b); return std::round(a * p) / p; }
    case WS_FN_TRUNCATE2: { const double p = std::pow(10.0, b); return std::trunc(a * p) / p; }
    case WS_FN_POW: return std::pow(a, b);
    case WS_FN_ATAN2: return std::atan2(a, b);
    case WS_FN_LOG_B: return (a <= 0 || b <= 0) ? nanv() : std::log(b) / std::log(a);
    case WS_FN_IDIV: return b == 0 ? nanv() : std::trunc(a / b);
    case WS_FN_ADD_MONTHS: return (double)addMonthsDays((int64_t)a, (int64_t)b);
    case WS_FN_DT_ADD_MONTHS: {
      const int64_t us = (int64_t)a, days = floorDiv(us, kUsPerDay);
      return (double)(addMonthsDays(days, (int64_t)b) * kUsPerDay + (us - days * kUsPerDay));
    }
    case WS_FN_DATE_TRUNC_MONTH: {
      int64_t y;
      unsigned m, d;
      civilFromDays((int64_t)a, y, m, d);
      return (double)daysFromCivil(y, b > 0 ? 1 : m, 1);
    }
  }
  return nanv();
}
double cmp3(int op, double a, double b) {
  if (isnan_(a) || isnan_(b)) return nanv();
  const bool r = op == 0 ? a == b : op == 1 ? a != b : op == 2 ? a < b : op == 3 ? a <= b : op == 4 ? a > b : a >= b;
  return r ? 1.0 : 0.0;
}
double and3(double a, double b) {
  if ((a == a && a == 0) || (b == b && b == 0)) return 0.0;
  if (isnan_(a) || isnan_(b)) return nanv();
  return 1.0;
}
double or3(double a, double b) {
  if ((a == a && a != 0) || (b == b && b != 0)) return 1.0;
  if (isnan_(a) || isnan_(b)) return nanv();
  return 0.0;
}
double insetD(const uint32_t* bits, int size, double x) {
  if (isnan_(x)) return x;
  const int64_t c = (int64_t)x;
  return (c >= 0 && c < size) ? (double)((bits[c >> 5] >> (c & 31)) & 1u) : 0.0;
}
int64_t insetI(const uint32_t* bits, int size, int64_t c) {
  return (c >= 0 && c < size) ? (int64_t)((bits[c >> 5] >> (c & 31)) & 1u) : 0;
}
double insortedD(const double* a, int n, double x) {
  if (isnan_(x)) return x;
  const double* p = std::lower_bound(a, a + n, x);
  return (p != a + n && *p == x) ? 1.0 : 0.0;
}
double dictmapD(const double* map, int size, double x) {
  if (isnan_(x)) return x;
  const int64_t c = (int64_t)x;
  return (c >= 0 && c < size) ? map[c] : nanv();
}
// checked int64 arithmetic (src/devtypes.h:197-215): wraps, and flags an overflow
int64_t iadd(int64_t a, int64_t b, int& f) {
  int64_t r;
  if (__builtin_add_overflow(a, b, &r)) f = 1;
  return r;
}
int64_t isub(int64_t a, int64_t b, int& f) {
  int64_t r;
  if (__builtin_sub_overflow(a, b, &r)) f = 1;
  return r;
}
int64_t imul(int64_t a, int64_t b, int& f) {
  int64_t r;
  if (__builtin_mul_overflow(a, b, &r)) f = 1;
  return r;
}

// ---------------------------------------------------------------- typed expression tree
struct Node {
  uint8_t op = 0;
  uint8_t isIntInstr = 0;
  uint16_t arg = 0;
  bool isInt = false;  // the node's static type (int64 or double)
  int kid[3] = {-1, -1, -1};
};
struct Tree {
  std::vector<Node> nodes;
  int root = -1;
};

// Rebuilds the expression tree from stack bytecode and types every node the way the reference's
// code generator does (src/jit.cu:113-273).
Tree buildTree(const ws_expr_env& env, ws_prog p) {
  Tree t;
  std::vector<int> st;
  auto pop = [&]() {
    if (st.empty()) throw std::runtime_error("malformed expression");
    const int v = st.back();
    st.pop_back();
    return v;
  };
  for (int pc = p.start; pc < p.start + p.len; ++pc) {
    const ws_instr in = env.code[pc];
    Node n;
    n.op = in.op;
    n.isIntInstr = in.isInt;
    n.arg = in.arg;
    switch (in.op) {
      case WS_OP_COL: {
        const int ty = env.cols[in.arg].t;
        n.isInt = ty == 0 || ty == 1;
        break;
      }
      case WS_OP_COLRAW: n.isInt = !(env.cols[in.arg].t == 6 && !in.isInt); break;
      case WS_OP_CONST: n.isInt = in.isInt != 0; break;
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL: case WS_OP_EQ: case WS_OP_NE: case WS_OP_LT: case WS_OP_LE:
      case WS_OP_GT: case WS_OP_GE: case WS_OP_AND: case WS_OP_OR: {
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[0]].isInt && t.nodes[n.kid[1]].isInt;
        break;
      }
      case WS_OP_DIV: case WS_OP_MOD: case WS_OP_NULLIF: case WS_OP_CALL2:
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = false;
        break;
      case WS_OP_COALESCE:
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[0]].isInt;
        break;
      case WS_OP_NEG: case WS_OP_NOT: case WS_OP_INSET: case WS_OP_YEAR:
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[0]].isInt;
        break;
      case WS_OP_ISNULL:
        n.kid[0] = pop();
        n.isInt = true;
        break;
      case WS_OP_CALL1: case WS_OP_DICTMAP: case WS_OP_INSORTED:
        n.kid[0] = pop();
        n.isInt = false;
        break;
      case WS_OP_SELECT:
        n.kid[2] = pop();
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[1]].isInt && t.nodes[n.kid[2]].isInt;
        break;
      case WS_OP_VDOT: case WS_OP_VEUC: n.isInt = false; break;
      default: throw std::runtime_error("unknown opcode");
    }
    t.nodes.push_back(n);
    st.push_back((int)t.nodes.size() - 1);
  }
  if (st.size() != 1) throw std::runtime_error("malformed expression");
  t.root = st[0];
  return t;
}

// Values of one node over a block of rows: int64 when the node is integer-typed, else double.
struct Vals {
  std::vector<int64_t> i;
  std::vector<double> d;
};

struct BlockEval {
  const ws_expr_env& env;
  const ws_col_view* cols;
  int ovf = 0;

  double asD(const Node& n, const Vals& v, int j) const { return n.isInt ? (double)v.i[j] : v.d[j]; }
  int64_t asI(const Node& n, const Vals& v, int j) const { return n.isInt ? v.i[j] : (int64_t)v.d[j]; }

  // Evaluates node `ni` of `t` for rows r0 .. r0+len-1 into out.
  void eval(const Tree& t, int ni, int64_t r0, int len, Vals& out) {
    const Node& n = t.nodes[ni];
    if (n.isInt) out.i.resize(len);
    else out.d.resize(len);
    Vals a, b, c;
    const Node* na = n.kid[0] >= 0 ? &t.nodes[n.kid[0]] : nullptr;
    const Node* nb = n.kid[1] >= 0 ? &t.nodes[n.kid[1]] : nullptr;
    const Node* nc = n.kid[2] >= 0 ? &t.nodes[n.kid[2]] : nullptr;
    if (na) eval(t, n.kid[0], r0, len, a);
    if (nb) eval(t, n.kid[1], r0, len, b);
    if (nc) eval(t, n.kid[2], r0, len, c);
    switch (n.op) {
      case WS_OP_COL: {
        const ws_col_view& cv = cols[n.arg];
        for (int j = 0; j < len; ++j) {
          const int64_t r = r0 + j;
          switch (cv.t) {
            case 0: case 1: out.i[j] = colInt(cv, r); break;
            case 2: out.d[j] = colDbl(cv, r); break;
            case 3: { const int64_t v = colInt(cv, r); out.d[j] = v == (int64_t)WS_NULL_I32 ? nanv() : (double)v; break; }
            case 4: { const int64_t v = colInt(cv, r); out.d[j] = v == WS_NULL_I64 ? nanv() : (double)v; break; }
            case 6: {
              const int64_t v = colInt(cv, r);
              out.d[j] = v == WS_NULL_I64 ? nanv() : (double)v / (double)(int64_t)pow10i(cv.scale);
              break;
            }
            default: out.d[j] = nanv(); break;
          }
        }
        break;
      }
      case WS_OP_COLRAW: {
        const ws_col_view& cv = cols[n.arg];
        for (int j = 0; j < len; ++j) {
          const int64_t v = colInt(cv, r0 + j);
          if (n.isInt) out.i[j] = v;
          else out.d[j] = v == WS_NULL_I64 ? nanv() : (double)v;
        }
        break;
      }
      case WS_OP_CONST:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = dbits(env.consts[n.arg]);
          else out.d[j] = env.consts[n.arg];
        }
        break;
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) {
            out.i[j] = n.op == WS_OP_ADD ? iadd(a.i[j], b.i[j], ovf) : n.op == WS_OP_SUB ? isub(a.i[j], b.i[j], ovf)
                                                                       : imul(a.i[j], b.i[j], ovf);
          } else {
            const double x = asD(*na, a, j), y = asD(*nb, b, j);
            out.d[j] = n.op == WS_OP_ADD ? x + y : n.op == WS_OP_SUB ? x - y : x * y;
          }
        }
        break;
      case WS_OP_DIV:
        for (int j = 0; j < len; ++j) {
          const double x = asD(*na, a, j), y = asD(*nb, b, j);
          out.d[j] = y == 0 ? nanv() : x / y;
        }
        break;
      case WS_OP_MOD:
        for (int j = 0; j < len; ++j) out.d[j] = std::fmod(asD(*na, a, j), asD(*nb, b, j));
        break;
      case WS_OP_NEG:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = (int64_t)(0ull - (uint64_t)a.i[j]);
          else out.d[j] = -a.d[j];
        }
        break;
      case WS_OP_EQ: case WS_OP_NE: case WS_OP_LT: case WS_OP_LE: case WS_OP_GT: case WS_OP_GE: {
        const int o = n.op - WS_OP_EQ;
        for (int j = 0; j < len; ++j) {
          if (n.isInt) {
            const int64_t x = a.i[j], y = b.i[j];
            out.i[j] = o == 0 ? x == y : o == 1 ? x != y : o == 2 ? x < y : o == 3 ? x <= y : o == 4 ? x > y : x >= y;
          } else {
            out.d[j] = cmp3(o, asD(*na, a, j), asD(*nb, b, j));
          }
        }
        break;
      }
      case WS_OP_AND: case WS_OP_OR:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = n.op == WS_OP_AND ? (a.i[j] != 0 && b.i[j] != 0) : (a.i[j] != 0 || b.i[j] != 0);
          else out.d[j] = n.op == WS_OP_AND ? and3(asD(*na, a, j), asD(*nb, b, j)) : or3(asD(*na, a, j), asD(*nb, b, j));
        }
        break;
      case WS_OP_NOT:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = a.i[j] == 0;
          else out.d[j] = isnan_(a.d[j]) ? a.d[j] : (a.d[j] == 0 ? 1.0 : 0.0);
        }
        break;
      case WS_OP_INSET:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = insetI(env.sets[n.arg], env.setSize[n.arg], a.i[j]);
          else out.d[j] = insetD(env.sets[n.arg], env.setSize[n.arg], a.d[j]);
        }
        break;
      case WS_OP_SELECT:
        for (int j = 0; j < len; ++j) {
          const bool cond = na->isInt ? a.i[j] != 0 : truthy(a.d[j]);
          if (n.isInt) out.i[j] = cond ? b.i[j] : c.i[j];
          else out.d[j] = cond ? asD(*nb, b, j) : asD(*nc, c, j);
        }
        break;
      case WS_OP_YEAR:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) {
            int64_t y;
            unsigned m, d;
            civilFromDays(a.i[j], y, m, d);
            out.i[j] = y;
          } else {
            out.d[j] = call1(WS_FN_DT_YEAR, call1(WS_FN_DATE_TO_DT, a.d[j]));
          }
        }
        break;
      case WS_OP_ISNULL:
        for (int j = 0; j < len; ++j) out.i[j] = na->isInt ? 0 : isnan_(a.d[j]);
        break;
      case WS_OP_COALESCE:
        for (int j = 0; j < len; ++j) {
          if (n.isInt) out.i[j] = a.i[j];
          else out.d[j] = isnan_(a.d[j]) ? asD(*nb, b, j) : a.d[j];
        }
        break;
      case WS_OP_NULLIF:
        for (int j = 0; j < len; ++j) {
          const double x = asD(*na, a, j), y = asD(*nb, b, j);
          out.d[j] = x == y ? nanv() : x;
        }
        break;
      case WS_OP_CALL1:
        for (int j = 0; j < len; ++j) out.d[j] = call1(n.arg, asD(*na, a, j));
        break;
      case WS_OP_CALL2:
        for (int j = 0; j < len; ++j) out.d[j] = call2(n.arg, asD(*na, a, j), asD(*nb, b, j));
        break;
      case WS_OP_DICTMAP:
        for (int j = 0; j < len; ++j) out.d[j] = dictmapD(env.maps[n.arg], env.mapSize[n.arg], asD(*na, a, j));
        break;
      case WS_OP_INSORTED:
        for (int j = 0; j < len; ++j) out.d[j] = insortedD(env.maps[n.arg], env.mapSize[n.arg], asD(*na, a, j));
        break;
      case WS_OP_VDOT: case WS_OP_VEUC: {
        const int slot = n.arg & 255, mi = n.arg >> 8;
        const float* v = (const float*)cols[slot].p;
        const double* q = env.maps[mi];
        const int dim = env.mapSize[mi];
        for (int j = 0; j < len; ++j) {
          const float* x = v + (r0 + j) * (int64_t)dim;
          if (isnan_(x[0])) {
            out.d[j] = nanv();
            continue;
          }
          float acc = 0;
          for (int i = 0; i < dim; ++i) {
            if (n.op == WS_OP_VDOT) acc += x[i] * (float)q[i];
            else {
              const float dd = x[i] - (float)q[i];
              acc += dd * dd;
            }
          }
          out.d[j] = n.op == WS_OP_VDOT ? (double)acc : std::sqrt((double)acc);
        }
        break;
      }
    }
  }
};

bool isDeleted(const uint32_t* del, int64_t r) { return del && ((del[r >> 5] >> (r & 31)) & 1u); }

// ---------------------------------------------------------------- aggregation
// One slot's exact accumulator.
struct Acc {
  i128 s = 0;       // integer SUM
  int64_t v = 0;    // COUNT / integer MIN / MAX
  double d = 0;     // double SUM / MIN / MAX
};
struct SlotKind {
  uint8_t op;
  bool isInt;  // exact integer accumulation
  uint8_t nul;  // aggNull: 3 / 4
};

struct Group {
  std::vector<Acc> acc;
};

struct KeyHash {
  size_t operator()(const std::vector<int64_t>& k) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int64_t x : k) {
      h ^= (uint64_t)x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
      h *= 0xff51afd7ed558ccdull;
    }
    return (size_t)h;
  }
};
using GroupMap = std::unordered_map<std::vector<int64_t>, Group, KeyHash>;

void initAcc(const std::vector<SlotKind>& sk, Group& g) {
  g.acc.resize(sk.size());
  for (size_t a = 0; a < sk.size(); ++a) {
    Acc& x = g.acc[a];
    if (sk[a].isInt) x.v = sk[a].op == WS_AGG_MIN ? kLLMax : sk[a].op == WS_AGG_MAX ? kLLMin : 0;
    else x.d = sk[a].op == WS_AGG_MIN ? INFINITY : sk[a].op == WS_AGG_MAX ? -INFINITY : 0.0;
  }
}
void mergeAcc(const std::vector<SlotKind>& sk, Group& into, const Group& from) {
  for (size_t a = 0; a < sk.size(); ++a) {
    Acc& x = into.acc[a];
    const Acc& y = from.acc[a];
    const uint8_t op = sk[a].op;
    if (op == WS_AGG_COUNT) { x.v += y.v; continue; }
    if (sk[a].isInt) {
      if (op == WS_AGG_SUM) x.s += y.s;
      else if (op == WS_AGG_MIN) x.v = std::min(x.v, y.v);
      else x.v = std::max(x.v, y.v);
    } else {
      if (op == WS_AGG_SUM) x.d += y.d;
      else if (op == WS_AGG_MIN) x.d = std::fmin(x.d, y.d);
      else x.d = std::fmax(x.d, y.d);
    }
  }
}

struct PlanTrees {
  bool hasWhere;
  Tree where;
  std::vector<Tree> keys;
  std::vector<Tree> aggs;  // empty tree for COUNT
  std::vector<SlotKind> kinds;
  std::vector<uint8_t> keyInt;
  bool hasDistinct = false;
  Tree distinct;
  bool distinctInt = false;
};

PlanTrees makeTrees(const ws_expr_env& env, const ws_agg_plan& plan) {
  PlanTrees p;
  p.hasWhere = plan.hasWhere;
  if (plan.hasWhere) p.where = buildTree(env, plan.where);
  for (int k = 0; k < plan.nkeys; ++k) {
    p.keys.push_back(buildTree(env, plan.keys[k]));
    p.keyInt.push_back(plan.keyInt[k]);
  }
  for (int a = 0; a < plan.naggs; ++a) {
    SlotKind s{plan.ops[a], plan.ops[a] == WS_AGG_COUNT || plan.aggInt[a] != 0, plan.aggNull[a]};
    p.kinds.push_back(s);
    if (plan.ops[a] == WS_AGG_COUNT || a == 0) p.aggs.emplace_back();
    else p.aggs.push_back(buildTree(env, plan.aggs[a]));
  }
  return p;
}

struct Result {
  int nk = 0, na = 0, ovf = 0;
  std::vector<std::vector<int64_t>> keys;
  std::vector<std::vector<std::pair<int64_t, int64_t>>> words;
};

// Integer value of an aggregate argument for row j of the block: the typed int64, or for a nullable
// integer column (aggNull) its raw stored value (NULL -> the slot's neutral element, src/kernels.cuh:66-70).
struct RowAgg {
  static bool intArg(const SlotKind& s, const Tree& t, const Vals& v, int j, const ws_col_view* cols, int64_t r,
                     int64_t& out) {
    if (s.nul) {
      const int64_t raw = colInt(cols[t.nodes[t.root].arg], r);
      const int64_t nul = s.nul == 3 ? (int64_t)WS_NULL_I32 : WS_NULL_I64;
      if (raw == nul) return false;  // skipped
      out = raw;
      return true;
    }
    const Node& n = t.nodes[t.root];
    out = n.isInt ? v.i[j] : (int64_t)v.d[j];
    return true;
  }
};

// Aggregates rows [r0, r1) of batch b into `map` (per-thread partial).
void aggRange(const ws_expr_env& env, const PlanTrees& pt, const ws_col_view* cols, const uint32_t* del, int64_t r0,
              int64_t r1, GroupMap& map, std::unordered_map<std::vector<int64_t>, std::unordered_set<int64_t>, KeyHash>* dist,
              int& ovf) {
  BlockEval ev{env, cols, 0};
  const int nk = (int)pt.keys.size(), na = (int)pt.kinds.size();
  Vals wv, dv;
  std::vector<Vals> kv(nk), av(na);
  std::vector<int64_t> key(nk);
  for (int64_t b0 = r0; b0 < r1; b0 += kBlock) {
    const int len = (int)std::min<int64_t>(kBlock, r1 - b0);
    if (pt.hasWhere) ev.eval(pt.where, pt.where.root, b0, len, wv);
    for (int k = 0; k < nk; ++k) ev.eval(pt.keys[k], pt.keys[k].root, b0, len, kv[k]);
    for (int a = 1; a < na; ++a)
      if (pt.kinds[a].op != WS_AGG_COUNT) ev.eval(pt.aggs[a], pt.aggs[a].root, b0, len, av[a]);
    if (pt.hasDistinct) ev.eval(pt.distinct, pt.distinct.root, b0, len, dv);
    for (int j = 0; j < len; ++j) {
      const int64_t r = b0 + j;
      if (isDeleted(del, r)) continue;
      if (pt.hasWhere) {
        const Node& wn = pt.where.nodes[pt.where.root];
        if (wn.isInt ? wv.i[j] == 0 : !truthy(wv.d[j])) continue;
      }
      for (int k = 0; k < nk; ++k) {
        const Node& kn = pt.keys[k].nodes[pt.keys[k].root];
        if (pt.keyInt[k]) {
          key[k] = kn.isInt ? kv[k].i[j] : (int64_t)kv[k].d[j];
        } else {
          double d = kn.isInt ? (double)kv[k].i[j] : kv[k].d[j];
          d = d + 0.0;  // -0.0 groups with 0.0
          if (isnan_(d)) d = nanv();
          key[k] = dbits(d);
        }
      }
      auto it = map.find(key);
      if (it == map.end()) {
        Group g;
        initAcc(pt.kinds, g);
        it = map.emplace(key, std::move(g)).first;
      }
      Group& g = it->second;
      for (int a = 0; a < na; ++a) {
        const SlotKind& s = pt.kinds[a];
        Acc& x = g.acc[a];
        if (s.op == WS_AGG_COUNT) { ++x.v; continue; }
        if (s.isInt) {
          int64_t v;
          if (!RowAgg::intArg(s, pt.aggs[a], av[a], j, cols, r, v)) continue;
          if (s.op == WS_AGG_SUM) x.s += v;
          else if (s.op == WS_AGG_MIN) x.v = std::min(x.v, v);
          else x.v = std::max(x.v, v);
        } else {
          const Node& an = pt.aggs[a].nodes[pt.aggs[a].root];
          const double v = an.isInt ? (double)av[a].i[j] : av[a].d[j];
          if (isnan_(v)) continue;
          if (s.op == WS_AGG_SUM) x.d += v;
          else if (s.op == WS_AGG_MIN) x.d = std::fmin(x.d, v);
          else x.d = std::fmax(x.d, v);
        }
      }
      if (dist) {
        const Node& dn = pt.distinct.nodes[pt.distinct.root];
        if (dn.isInt) (*dist)[key].insert(dv.i[j]);
        else if (!isnan_(dv.d[j])) {
          double d = dv.d[j] + 0.0;
          (*dist)[key].insert(dbits(d));
        } else {
          (*dist)[key];  // the group exists; NULL is not counted
        }
      }
    }
  }
  ovf |= ev.ovf;
}

struct WorkItem {
  int b;
  int64_t r0, r1;
};

std::vector<WorkItem> splitWork(int nb, const int64_t* bn, int nthreads) {
  int64_t total = 0;
  for (int b = 0; b < nb; ++b) total += bn[b];
  const int64_t chunk = std::max<int64_t>(1 << 16, (total + nthreads * 4 - 1) / std::max(1, nthreads * 4));
  std::vector<WorkItem> w;
  for (int b = 0; b < nb; ++b)
    for (int64_t r = 0; r < bn[b]; r += chunk) w.push_back({b, r, std::min(bn[b], r + chunk)});
  return w;
}

template <class F>
void parallel(int nthreads, int nitems, F f) {
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  const int nt = std::max(1, std::min(nthreads, nitems));
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (int i; (i = next.fetch_add(1)) < nitems;) f(t, i);
    });
  for (auto& x : th) x.join();
}

int runAggregate(const ws_expr_env* env, const ws_agg_plan* plan, const ws_prog* distinct, int distinctInt, int nb,
                 const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int nthreads,
                 ws_oracle_result** out) {
  PlanTrees pt = makeTrees(*env, *plan);
  if (distinct) {
    pt.hasDistinct = true;
    pt.distinct = buildTree(*env, *distinct);
    pt.distinctInt = distinctInt;
  }
  nthreads = std::max(1, nthreads);
  const std::vector<WorkItem> work = splitWork(nb, bn, nthreads);
  const int nt = std::max(1, std::min<int>(nthreads, (int)work.size()));
  std::vector<GroupMap> maps(nt);
  using DistMap = std::unordered_map<std::vector<int64_t>, std::unordered_set<int64_t>, KeyHash>;
  std::vector<DistMap> dists(nt);
  std::vector<int> ovfs(nt, 0);
  parallel(nt, (int)work.size(), [&](int t, int i) {
    const WorkItem& w = work[i];
    aggRange(*env, pt, bcols + (int64_t)w.b * ncols, bdel ? bdel[w.b] : nullptr, w.r0, w.r1, maps[t],
             distinct ? &dists[t] : nullptr, ovfs[t]);
  });
  GroupMap all = std::move(maps[0]);
  for (int t = 1; t < nt; ++t)
    for (auto& kv : maps[t]) {
      auto it = all.find(kv.first);
      if (it == all.end()) all.emplace(kv.first, std::move(kv.second));
      else mergeAcc(pt.kinds, it->second, kv.second);
    }
  DistMap dall;
  if (distinct) {
    dall = std::move(dists[0]);
    for (int t = 1; t < nt; ++t)
      for (auto& kv : dists[t]) dall[kv.first].insert(kv.second.begin(), kv.second.end());
  }
  auto* r = new Result();
  r->nk = plan->nkeys;
  r->na = plan->naggs + (distinct ? 1 : 0);
  for (int t = 0; t < nt; ++t) r->ovf |= ovfs[t];
  if (plan->nkeys == 0 && all.empty()) {  // no rows: the identities
    Group g;
    initAcc(pt.kinds, g);
    all.emplace(std::vector<int64_t>{}, std::move(g));
  }
  std::vector<std::vector<int64_t>> order;
  for (auto& kv : all) order.push_back(kv.first);
  std::sort(order.begin(), order.end());
  for (auto& k : order) {
    const Group& g = all[k];
    std::vector<std::pair<int64_t, int64_t>> w(r->na);
    for (int a = 0; a < plan->naggs; ++a) {
      const SlotKind& s = pt.kinds[a];
      const Acc& x = g.acc[a];
      if (s.op == WS_AGG_COUNT) w[a] = {x.v, 0};
      else if (s.isInt && s.op == WS_AGG_SUM) w[a] = {(int64_t)(uint64_t)x.s, (int64_t)(x.s >> 64)};
      else if (s.isInt) w[a] = {x.v, 0};
      else w[a] = {dbits(x.d), 0};
    }
    if (distinct) w[plan->naggs] = {(int64_t)dall[k].size(), 0};
    r->keys.push_back(k);
    r->words.push_back(std::move(w));
  }
  *out = (ws_oracle_result*)r;
  return 0;
}

}  // namespace

extern "C" {

// Table::encodeColumn (src/storage.cu:1093-1192) restated: the engine's encoding of one segment column
// (ptype 0 I32, 1 I64, 2 F64).  Returns enc (0: raw) and, when cap allows, the bytes in out.
int ws_oracle_encode_column_engine(const void* src, int ptype, int64_t n, uint8_t* out, int64_t cap, int64_t* bytes) {
  *bytes = 0;
  if (n < 1024) return 0;
  std::vector<uint8_t> o;
  int e = 0;
  if (ptype == 0 || ptype == 1) {
    const bool i32 = ptype == 0;
    const long long nul = i32 ? (long long)WS_NULL_I32 : (long long)WS_NULL_I64;
    auto at = [&](int64_t i) { return i32 ? (long long)((const int32_t*)src)[i] : (long long)((const int64_t*)src)[i]; };
    long long mn = LLONG_MAX, mx = LLONG_MIN;
    for (int64_t i = 0; i < n; ++i) {
      const long long v = at(i);
      if (v == nul) continue;
      mn = std::min(mn, v), mx = std::max(mx, v);
    }
    if (mn > mx) mn = mx = 0;
    const unsigned long long range = (unsigned long long)mx - (unsigned long long)mn;
    e = range < 0xFFull ? 1 : range < 0xFFFFull ? 2 : (!i32 && range < 0xFFFFFFFFull) ? 3 : 0;
    if (!e) return 0;
    const int w = e == 1 ? 1 : e == 2 ? 2 : 4;
    o.assign(16 + (size_t)n * w + 16, 0);
    memcpy(o.data(), &mn, 8);
    for (int64_t i = 0; i < n; ++i) {
      const long long v = at(i);
      const unsigned long long c = v == nul ? ~0ull : (unsigned long long)v - (unsigned long long)mn;
      if (w == 1) o[16 + i] = (uint8_t)c;
      else if (w == 2) { const uint16_t c2 = (uint16_t)c; memcpy(&o[16 + 2 * i], &c2, 2); }
      else { const uint32_t c4 = (uint32_t)c; memcpy(&o[16 + 4 * i], &c4, 4); }
    }
  } else if (ptype == 2) {
    const double* x = (const double*)src;
    std::unordered_map<uint64_t, uint8_t> dict;
    std::vector<double> vals;
    bool many = false;
    for (int64_t i = 0; i < n && !many; ++i) {
      uint64_t b;
      memcpy(&b, &x[i], 8);
      if (dict.count(b)) continue;
      if (dict.size() == 255) { many = true; break; }
      dict.emplace(b, (uint8_t)dict.size());
      vals.push_back(x[i]);
    }
    if (!many) {
      e = 4;
      o.assign(16 + 256 * 8 + (size_t)n + 16, 0);
      memcpy(o.data() + 16, vals.data(), vals.size() * 8);
      for (int64_t i = 0; i < n; ++i) {
        uint64_t b;
        memcpy(&b, &x[i], 8);
        o[16 + 256 * 8 + i] = dict[b];
      }
    } else {
      double p = 1.0;
      for (int s = 0; s <= 4; ++s, p *= 10.0) {
        long long mn = LLONG_MAX, mx = LLONG_MIN;
        bool ok = true;
        for (int64_t i = 0; i < n && ok; ++i) {
          if (x[i] != x[i]) continue;
          const double y = x[i] * p;
          if (!(std::fabs(y) < 4e15)) { ok = false; break; }
          const long long k = std::llround(y);
          if ((double)k / p != x[i]) { ok = false; break; }
          mn = std::min(mn, k), mx = std::max(mx, k);
        }
        if (!ok) continue;
        if (mn > mx) mn = mx = 0;
        const unsigned long long range = (unsigned long long)(mx - mn);
        e = range < 0xFFFFull ? 5 : range < 0xFFFFFFFFull ? 6 : 0;
        if (!e) return 0;
        const int w = e == 5 ? 2 : 4;
        o.assign(16 + (size_t)n * w + 16, 0);
        memcpy(o.data(), &mn, 8);
        memcpy(o.data() + 8, &p, 8);
        for (int64_t i = 0; i < n; ++i) {
          const unsigned long long c = x[i] != x[i] ? ~0ull : (unsigned long long)(std::llround(x[i] * p) - mn);
          if (w == 2) { const uint16_t c2 = (uint16_t)c; memcpy(&o[16 + 2 * i], &c2, 2); }
          else { const uint32_t c4 = (uint32_t)c; memcpy(&o[16 + 4 * i], &c4, 4); }
        }
        break;
      }
      if (!e) return 0;
    }
  }
  *bytes = (int64_t)o.size();
  if (out && cap >= (int64_t)o.size()) memcpy(out, o.data(), o.size());
  return e;
}

// Static type of an expression (1 = int64, 0 = double), as buildTree types it; -1 when malformed.
int ws_oracle_prog_is_int(const ws_expr_env* env, ws_prog p) {
  try {
    const Tree t = buildTree(*env, p);
    return t.nodes[t.root].isInt ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

double ws_oracle_eval(const ws_expr_env* env, const ws_col_view* cols, ws_prog prog, int64_t row, int64_t* ival,
                      int* is_int, int* ovf) {
  Tree t = buildTree(*env, prog);
  BlockEval ev{*env, cols, 0};
  Vals v;
  ev.eval(t, t.root, row, 1, v);
  const Node& n = t.nodes[t.root];
  if (ovf) *ovf = ev.ovf;
  if (is_int) *is_int = n.isInt;
  if (n.isInt) {
    if (ival) *ival = v.i[0];
    return (double)v.i[0];
  }
  if (ival) *ival = (int64_t)v.d[0];
  return v.d[0];
}

int ws_oracle_aggregate(const ws_expr_env* env, const ws_agg_plan* plan, int nb, const int64_t* bn,
                        const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int nthreads,
                        ws_oracle_result** out) {
  try {
    return runAggregate(env, plan, nullptr, 0, nb, bn, bdel, bcols, ncols, nthreads, out);
  } catch (const std::exception&) {
    return 1;
  }
}

int ws_oracle_aggregate_distinct(const ws_expr_env* env, const ws_agg_plan* plan, ws_prog distinct, int distinct_int,
                                 int nb, const int64_t* bn, const uint32_t* const* bdel, const ws_col_view* bcols,
                                 int ncols, int nthreads, ws_oracle_result** out) {
  try {
    return runAggregate(env, plan, &distinct, distinct_int, nb, bn, bdel, bcols, ncols, nthreads, out);
  } catch (const std::exception&) {
    return 1;
  }
}

int64_t ws_oracle_ngroups(const ws_oracle_result* r) { return (int64_t)((const Result*)r)->keys.size(); }
int ws_oracle_nkeys(const ws_oracle_result* r) { return ((const Result*)r)->nk; }
int ws_oracle_naggs(const ws_oracle_result* r) { return ((const Result*)r)->na; }
int ws_oracle_overflow(const ws_oracle_result* r) { return ((const Result*)r)->ovf; }
void ws_oracle_keys(const ws_oracle_result* r, int64_t* keys) {
  const Result* x = (const Result*)r;
  for (size_t g = 0; g < x->keys.size(); ++g)
    for (int k = 0; k < x->nk; ++k) keys[g * x->nk + k] = x->keys[g][k];
}
void ws_oracle_words(const ws_oracle_result* r, int64_t* words) {
  const Result* x = (const Result*)r;
  for (size_t g = 0; g < x->words.size(); ++g)
    for (int a = 0; a < x->na; ++a) {
      words[(g * x->na + a) * 2] = x->words[g][a].first;
      words[(g * x->na + a) * 2 + 1] = x->words[g][a].second;
    }
}
void ws_oracle_free(ws_oracle_result* r) { delete (Result*)r; }

int64_t ws_oracle_select(const ws_expr_env* env, int has_where, ws_prog where, int nb, const int64_t* bn,
                         const uint32_t* const* bdel, const ws_col_view* bcols, int ncols, int nthreads,
                         int32_t* idx, int64_t* per_batch) {
  Tree t;
  if (has_where) t = buildTree(*env, where);
  std::vector<int64_t> boff(nb + 1, 0);
  for (int b = 0; b < nb; ++b) boff[b + 1] = boff[b] + bn[b];
  const std::vector<WorkItem> work = splitWork(nb, bn, std::max(1, nthreads));
  std::vector<std::vector<int32_t>> sel(work.size());
  parallel(std::max(1, nthreads), (int)work.size(), [&](int, int i) {
    const WorkItem& w = work[i];
    BlockEval ev{*env, bcols + (int64_t)w.b * ncols, 0};
    const uint32_t* del = bdel ? bdel[w.b] : nullptr;
    Vals v;
    for (int64_t b0 = w.r0; b0 < w.r1; b0 += kBlock) {
      const int len = (int)std::min<int64_t>(kBlock, w.r1 - b0);
      if (has_where) ev.eval(t, t.root, b0, len, v);
      for (int j = 0; j < len; ++j) {
        if (isDeleted(del, b0 + j)) continue;
        if (has_where) {
          const Node& n = t.nodes[t.root];
          if (n.isInt ? v.i[j] == 0 : !truthy(v.d[j])) continue;
        }
        sel[i].push_back((int32_t)(boff[w.b] + b0 + j));
      }
    }
  });
  int64_t m = 0;
  if (per_batch)
    for (int b = 0; b < nb; ++b) per_batch[b] = 0;
  for (size_t i = 0; i < work.size(); ++i) {
    if (idx) memcpy(idx + m, sel[i].data(), sel[i].size() * 4);
    if (per_batch) per_batch[work[i].b] += (int64_t)sel[i].size();
    m += (int64_t)sel[i].size();
  }
  return m;
}

// Join keys (src/gpu.cu:180-202): I32 views (t 0 / 3) widen to int64 and their sentinel is NULL, I64
// views (t 1 / 4) use theirs; NULL never matches.
static bool joinKey(const ws_col_view& c, int64_t r, int64_t& k) {
  if (c.t == 0 || c.t == 3) {
    const int32_t v = ((const int32_t*)c.p)[r];
    k = v;
    return v != WS_NULL_I32;
  }
  if (c.t == 1 || c.t == 4) {
    k = ((const int64_t*)c.p)[r];
    return k != WS_NULL_I64;
  }
  const double d = ((const double*)c.p)[r];
  k = (int64_t)d;
  return d == d;
}

int64_t ws_oracle_hash_join(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int nthreads,
                            int32_t* out_build, int32_t* out_probe) {
  std::unordered_map<int64_t, std::vector<int32_t>> table;
  table.reserve((size_t)nb * 2);
  for (int64_t i = 0; i < nb; ++i) {
    int64_t k;
    if (joinKey(build_key, i, k)) table[k].push_back((int32_t)i);
  }
  for (auto& kv : table) std::sort(kv.second.begin(), kv.second.end());
  nthreads = std::max(1, nthreads);
  const int64_t chunk = std::max<int64_t>(1 << 16, (np + nthreads * 4 - 1) / (nthreads * 4));
  const int nchunks = (int)((np + chunk - 1) / chunk);
  std::vector<int64_t> cnt(nchunks, 0);
  parallel(nthreads, nchunks, [&](int, int c) {
    int64_t n = 0;
    for (int64_t j = c * chunk; j < std::min(np, (c + 1) * chunk); ++j) {
      int64_t k;
      if (!joinKey(probe_key, j, k)) continue;
      auto it = table.find(k);
      if (it != table.end()) n += (int64_t)it->second.size();
    }
    cnt[c] = n;
  });
  std::vector<int64_t> off(nchunks + 1, 0);
  for (int c = 0; c < nchunks; ++c) off[c + 1] = off[c] + cnt[c];
  if (out_build && out_probe)
    parallel(nthreads, nchunks, [&](int, int c) {
      int64_t o = off[c];
      for (int64_t j = c * chunk; j < std::min(np, (c + 1) * chunk); ++j) {
        int64_t k;
        if (!joinKey(probe_key, j, k)) continue;
        auto it = table.find(k);
        if (it == table.end()) continue;
        for (int32_t b : it->second) {
          out_build[o] = b;
          out_probe[o] = (int32_t)j;
          ++o;
        }
      }
    });
  return off[nchunks];
}

void ws_oracle_gather_multi(const ws_col_view* src, const int64_t* boff, int nb, int ptype, int esize,
                            const int32_t* idx, int64_t m, void* dst) {
  for (int64_t j = 0; j < m; ++j) {
    const int64_t g = idx[j];
    const int b = (int)(std::upper_bound(boff, boff + nb, g) - boff) - 1;
    const ws_col_view& v = src[b];
    const int64_t r = g - boff[b];
    if (v.enc) {
      ws_col_view w = v;
      w.t = ptype == WS_PT_I32 ? 3 : ptype == WS_PT_I64 ? 4 : 2;
      if (ptype == WS_PT_F64) ((double*)dst)[j] = colDbl(w, r);
      else if (ptype == WS_PT_I32) ((int32_t*)dst)[j] = (int32_t)colInt(w, r);
      else ((int64_t*)dst)[j] = colInt(w, r);
    } else {
      memcpy((uint8_t*)dst + j * esize, (const uint8_t*)v.p + r * esize, esize);
    }
  }
}


/* ---- outer join, sort permutation, evaluation at rows (restatements of src/gpu.cu:1197-1293,
 * :1323-1361, :862-888, :1011-1019) */

int64_t ws_oracle_hash_join_outer(ws_col_view build_key, int64_t nb, ws_col_view probe_key, int64_t np, int full,
                                  int32_t* out_build, int32_t* out_probe) {
  std::unordered_map<int64_t, std::vector<int32_t>> table;
  table.reserve((size_t)nb * 2);
  for (int64_t i = 0; i < nb; ++i) {
    int64_t k;
    if (joinKey(build_key, i, k)) table[k].push_back((int32_t)i);
  }
  for (auto& kv : table) std::sort(kv.second.begin(), kv.second.end());
  std::vector<uint8_t> matched(full ? (size_t)nb : 0, 0);
  int64_t o = 0;
  auto emit = [&](int32_t b, int32_t p) {
    if (out_build) out_build[o] = b, out_probe[o] = p;
    ++o;
  };
  for (int64_t j = 0; j < np; ++j) {  // probe order: matches, or one pair with build row -1
    int64_t k;
    auto it = joinKey(probe_key, j, k) ? table.find(k) : table.end();
    if (it == table.end()) {
      emit(-1, (int32_t)j);
      continue;
    }
    for (int32_t b : it->second) {
      emit(b, (int32_t)j);
      if (full) matched[b] = 1;
    }
  }
  if (full)
    for (int64_t i = 0; i < nb; ++i)
      if (!matched[i]) emit((int32_t)i, -1);
  return o;
}

static uint64_t orderKeyOf(double v, bool desc) {
  if (v != v) v = -INFINITY;  // NULL first (ascending)
  if (v == 0.0) v = 0.0;
  uint64_t b;
  memcpy(&b, &v, 8);
  b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
  return desc ? ~b : b;
}

void ws_oracle_sort_perm(const double* const* keys, const int* desc, int nkeys, int64_t m, int32_t* perm) {
  std::vector<std::vector<uint64_t>> k(nkeys, std::vector<uint64_t>((size_t)m));
  for (int c = 0; c < nkeys; ++c)
    for (int64_t i = 0; i < m; ++i) k[c][i] = orderKeyOf(keys[c][i], desc[c] != 0);
  for (int64_t i = 0; i < m; ++i) perm[i] = (int32_t)i;
  std::stable_sort(perm, perm + m, [&](int32_t a, int32_t b) {
    for (int c = 0; c < nkeys; ++c)
      if (k[c][a] != k[c][b]) return k[c][a] < k[c][b];
    return false;
  });
}

void ws_oracle_eval_at(const ws_expr_env* env, const ws_col_view* cols, ws_prog prog, const int32_t* idx, int64_t m,
                       int as_int, void* out, int* ovf) {
  Tree t = buildTree(*env, prog);
  const Node& n = t.nodes[t.root];
  const ws_instr in0 = env->code[prog.start];
  const bool single = prog.len == 1 && in0.op == WS_OP_COL && cols[in0.arg].t != 2;
  BlockEval ev{*env, cols, 0};
  for (int64_t j = 0; j < m; ++j) {
    const int64_t r = idx ? idx[j] : j;
    Vals v;
    ev.eval(t, t.root, r, 1, v);
    if (!as_int) {
      ((double*)out)[j] = n.isInt ? (double)v.i[0] : v.d[0];
      continue;
    }
    int64_t o;
    if (single) {  // the column's stored value; INT NULL widened to the BIGINT NULL
      const ws_col_view& c = cols[in0.arg];
      int64_t x = colInt(c, r);
      if ((c.t == 0 || c.t == 3) && x == (int64_t)(int32_t)0x80000000) x = (int64_t)0x8000000000000000ull;
      o = x;
    } else if (n.isInt) {
      o = v.i[0];
    } else {
      o = v.d[0] != v.d[0] ? (int64_t)0x8000000000000000ull : llround(v.d[0]);
    }
    ((int64_t*)out)[j] = o;
  }
  if (ovf) *ovf = ev.ovf;
}

}  // extern "C"
