// On-device interpreter evaluator: runs the engine's expression bytecode, typed on the host exactly as
// the code generator types it (ws_plan.cpp), so interpreted and compiled plans compute the same values.
// Used when codegen is off (jit mode OFF) or a plan failed to compile; generated evaluators are the
// fast path.
#pragma once
#include "ws_kern.cuh"

namespace ws {

// Stored integer of any integer view (raw or encoded), the type's NULL sentinel for NULL.
WS_DI i64 colIntAt(const ws_col_view& v, i64 r) {
  const bool i32 = v.t == 0 || v.t == 3;
  if (!v.enc) return i32 ? (i64)__ldg((const int*)v.p + r) : __ldg((const i64*)v.p + r);
  const i64 nul = i32 ? (i64)WS_NULL_I32 : (i64)WS_NULL_I64;
  if (v.enc >= 7) {
    i64 o[4];
    load4encView(o, &v, r, nul, 1);
    return o[0];
  }
  const ColRef c = resolveCol(v);
  unsigned code;
  if (c.enc == 1) {
    code = __ldg(c.d + r);
    return code == 0xffu ? nul : c.base + (i64)code;
  }
  if (c.enc == 2) {
    code = __ldg((const unsigned short*)c.d + r);
    return code == 0xffffu ? nul : c.base + (i64)code;
  }
  code = __ldg((const unsigned*)c.d + r);
  return code == 0xffffffffu ? nul : c.base + (i64)code;
}
WS_DI double colDblAt(const ws_col_view& v, i64 r) {
  if (!v.enc) return __ldg((const double*)v.p + r);
  const ColRef c = resolveCol(v);
  if (c.enc == 4) return __ldg(c.dict + __ldg(c.d + r));
  const unsigned code = c.enc == 5 ? (unsigned)__ldg((const unsigned short*)c.d + r) : __ldg((const unsigned*)c.d + r);
  const unsigned nulc = c.enc == 5 ? 0xffffu : 0xffffffffu;
  return code == nulc ? nanv() : (double)(c.base + (i64)code) / c.p10;
}
WS_DI double pow10d(int s) {
  double p = 1;
  for (int i = 0; i < s; ++i) p *= 10;
  return p;
}

union Word {
  i64 i;
  double d;
};
WS_DI double asD(Word w, uint8_t isInt) { return isInt ? (double)w.i : w.d; }

// Runs one typed program for row r of the batch whose views are cv.
static __device__ __noinline__ Word vmRun(const TInstr* code, int start, int len, const ws_col_view* cv, i64 r,
                                   const EnvK& env) {
  Word st[WS_MAX_STACK];
  int sp = 0;
  for (int pc = start; pc < start + len; ++pc) {
    const TInstr in = code[pc];
    Word out;
    switch (in.op) {
      case WS_OP_COL: {
        const ws_col_view& v = cv[in.arg];
        switch (v.t) {
          case 0: case 1: out.i = colIntAt(v, r); break;
          case 2: out.d = colDblAt(v, r); break;
          case 3: out.d = nullIfI32(colIntAt(v, r)); break;
          case 4: out.d = nullIfI64(colIntAt(v, r)); break;
          case 6: out.d = decOf(colIntAt(v, r), pow10d(v.scale)); break;
          default: out.d = nanv(); break;
        }
        st[sp++] = out;
        continue;
      }
      case WS_OP_COLRAW: {
        const i64 v = colIntAt(cv[in.arg], r);
        if (in.rInt) out.i = v;
        else out.d = nullIfI64(v);
        st[sp++] = out;
        continue;
      }
      case WS_OP_CONST:
        out.d = env.consts[in.arg];  // an integer literal's bits are its int64
        st[sp++] = out;
        continue;
      case WS_OP_VDOT: case WS_OP_VEUC: {
        const int slot = in.arg & 255, m = in.arg >> 8;
        out.d = vecD(in.op == WS_OP_VDOT, (const float*)cv[slot].p, r, env.maps[m], env.mapSize[m]);
        st[sp++] = out;
        continue;
      }
      default: break;
    }
    // operators: pop operands (a = first pushed)
    Word a, b, c;
    if (in.op == WS_OP_SELECT) {
      c = st[--sp];
      b = st[--sp];
      a = st[--sp];
    } else if (in.op == WS_OP_NEG || in.op == WS_OP_NOT || in.op == WS_OP_INSET || in.op == WS_OP_YEAR ||
               in.op == WS_OP_ISNULL || in.op == WS_OP_CALL1 || in.op == WS_OP_DICTMAP || in.op == WS_OP_INSORTED) {
      a = st[--sp];
    } else {
      b = st[--sp];
      a = st[--sp];
    }
    switch (in.op) {
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL:
        if (in.rInt) {
          out.i = in.op == WS_OP_ADD ? iaddc(a.i, b.i, env.ovf) : in.op == WS_OP_SUB ? isubc(a.i, b.i, env.ovf)
                                                                  : imulc(a.i, b.i, env.ovf);
        } else {
          const double x = asD(a, in.aInt), y = asD(b, in.bInt);
          out.d = in.op == WS_OP_ADD ? x + y : in.op == WS_OP_SUB ? x - y : x * y;
        }
        break;
      case WS_OP_DIV: out.d = divz(asD(a, in.aInt), asD(b, in.bInt)); break;
      case WS_OP_MOD: out.d = fmod(asD(a, in.aInt), asD(b, in.bInt)); break;
      case WS_OP_NEG:
        if (in.rInt) out.i = (i64)(0ull - (u64)a.i);
        else out.d = -a.d;
        break;
      case WS_OP_EQ: case WS_OP_NE: case WS_OP_LT: case WS_OP_LE: case WS_OP_GT: case WS_OP_GE: {
        const int o = in.op - WS_OP_EQ;
        if (in.rInt) {
          const i64 x = a.i, y = b.i;
          out.i = o == 0 ? x == y : o == 1 ? x != y : o == 2 ? x < y : o == 3 ? x <= y : o == 4 ? x > y : x >= y;
        } else {
          out.d = cmp3(o, asD(a, in.aInt), asD(b, in.bInt));
        }
        break;
      }
      case WS_OP_AND: case WS_OP_OR:
        if (in.rInt) out.i = in.op == WS_OP_AND ? (a.i != 0 && b.i != 0) : (a.i != 0 || b.i != 0);
        else out.d = in.op == WS_OP_AND ? and3(asD(a, in.aInt), asD(b, in.bInt)) : or3(asD(a, in.aInt), asD(b, in.bInt));
        break;
      case WS_OP_NOT:
        if (in.rInt) out.i = a.i == 0;
        else out.d = not3(a.d);
        break;
      case WS_OP_INSET:
        if (in.rInt) out.i = insetI(env.sets[in.arg], env.setSize[in.arg], a.i);
        else out.d = insetD(env.sets[in.arg], env.setSize[in.arg], a.d);
        break;
      case WS_OP_SELECT: {
        const bool cond = in.aInt ? a.i != 0 : truthy(a.d);
        if (in.rInt) out.i = cond ? b.i : c.i;
        else out.d = cond ? asD(b, in.bInt) : asD(c, in.cInt);
        break;
      }
      case WS_OP_YEAR:
        if (in.rInt) out.i = yearOf(a.i);
        else out.d = yearD(a.d);
        break;
      case WS_OP_ISNULL: out.i = in.aInt ? 0 : (a.d != a.d); break;
      case WS_OP_COALESCE:
        if (in.rInt) out.i = a.i;
        else out.d = coalesce2(a.d, asD(b, in.bInt));
        break;
      case WS_OP_NULLIF: out.d = nullif2(asD(a, in.aInt), asD(b, in.bInt)); break;
      case WS_OP_CALL1: out.d = call1(in.arg, asD(a, in.aInt)); break;
      case WS_OP_CALL2: out.d = call2(in.arg, asD(a, in.aInt), asD(b, in.bInt)); break;
      case WS_OP_DICTMAP: out.d = dictmapD(env.maps[in.arg], env.mapSize[in.arg], asD(a, in.aInt)); break;
      case WS_OP_INSORTED: out.d = insortedD(env.maps[in.arg], env.mapSize[in.arg], asD(a, in.aInt)); break;
      default: out.d = nanv(); break;
    }
    st[sp++] = out;
  }
  return st[0];
}

struct InterpEv {
  static constexpr int NK = WS_INTERP_KEYS, NA = WS_INTERP_AGGS, RW = 1 + 2 * WS_INTERP_AGGS, FRW = WS_INTERP_AGGS;
  static constexpr int PRIV_MIN_BLOCKS = 1;  // the VM needs its registers
  static constexpr int HASH_MULTI_MIN_BLOCKS = 1;
  static constexpr bool STAGED = false;
  static constexpr int STAGE_BYTES = 0;
  const Launch& L;
  const ws_col_view* cv = nullptr;
  i64 r0 = 0;
  bool fastOk = false;
  __device__ InterpEv(const Launch& l) : L(l) {}
  WS_DI void bind(const Launch&, int b) { cv = L.cols + (i64)b * L.ncols; }
  WS_DI void load(i64 r, bool, int) { r0 = r; }
  WS_DI void prep(int, bool) {}
  WS_DI void finish() {}  // the VM raises overflow itself
  WS_DI int nk() const { return L.nkeys; }
  WS_DI int na() const { return L.naggs; }
  WS_DI int rowWords() const { return L.rowWords; }
  WS_DI int kind(int a) const { return __ldg(L.kinds + a); }
  WS_DI int woff(int a) const { return __ldg(L.woff + a); }
  WS_DI int fwoff(int a) const { return __ldg(L.fwoff + a); }
  WS_DI int fastWords() const { return L.fastWords; }
  WS_DI bool keyInt(int k) const { return __ldg(L.keyInt + k) != 0; }
  WS_DI Word run(const int (&p)[2], int i) const { return vmRun(L.progs->code, p[0], p[1], cv, r0 + i, L.env); }
  WS_DI bool resInt(const int (&p)[2]) const { return L.progs->code[p[0] + p[1] - 1].rInt != 0; }
  WS_DI bool where(int i) const {
    if (L.progs->where[1] == 0) return true;
    const Word w = run(L.progs->where, i);
    return resInt(L.progs->where) ? w.i != 0 : truthy(w.d);
  }
  WS_DI i64 ikey(int k, int i) const {
    const Word w = run(L.progs->keys[k], i);
    return resInt(L.progs->keys[k]) ? w.i : (i64)w.d;
  }
  WS_DI double dkey(int k, int i) const {
    const Word w = run(L.progs->keys[k], i);
    return resInt(L.progs->keys[k]) ? (double)w.i : w.d;
  }
  WS_DI bool ival(int a, int i, i64& v) const {
    const uint8_t nul = __ldg(L.aggNull + a);
    if (nul) {  // a nullable integer column read raw; its NULL sentinel is skipped
      const int col = L.progs->code[L.progs->aggs[a][0]].arg;
      v = colIntAt(cv[col], r0 + i);
      return v != (nul == 3 ? (i64)WS_NULL_I32 : (i64)WS_NULL_I64);
    }
    const Word w = run(L.progs->aggs[a], i);
    v = resInt(L.progs->aggs[a]) ? w.i : (i64)w.d;
    return true;
  }
  WS_DI double dval(int a, int i) const {
    const Word w = run(L.progs->aggs[a], i);
    return resInt(L.progs->aggs[a]) ? (double)w.i : w.d;
  }
};

}  // namespace ws
