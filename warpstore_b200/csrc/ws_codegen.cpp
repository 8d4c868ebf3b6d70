// Per-query code generation and the plan cache (the engine's jit layer: src/jit.h, src/jit.cu).
//
// A plan's expressions (filter, keys, aggregate arguments) are translated from the engine's bytecode
// into a typed C++ evaluator (struct QEv) that loads 4 rows per thread with vector loads and computes
// each expression in registers; the scan kernel bodies of ws_kern.cuh are instantiated with it and the
// module is compiled by NVRTC for the device's architecture (sm_100a on B200).  Literal values are not
// part of the source (they are read from the launch's constants), so one query shape compiles once.
// Compiled images are cached in memory (key: kernel kind + evaluator source) and, with a cache
// directory, on disk (key: NVRTC version + options + full source; the file carries a checksum).
#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <set>
#include <sstream>
#include <thread>

#include "ws_internal.h"
#include "ws_jit_sources.h"  // generated at build time: ws_types.h, ws_dev.cuh, ws_kern.cuh as strings

namespace ws {

namespace {

std::atomic<int> gDefaultMode{WS_JIT_ON};
thread_local int tMode = -1;
std::mutex gMu;
std::map<std::string, std::shared_ptr<ws_jit_program>> gCache;
std::vector<std::shared_ptr<ws_jit_program>> gById;
std::string gDiskDir;
thread_local std::string tSql;
thread_local ws_jit_query_info tInfo;
thread_local std::vector<ws_jit_program*> tUsed;
thread_local std::vector<int> tLastIds;  // plans used by the calling thread's last ended query

int jitMode() { return tMode >= 0 ? tMode : gDefaultMode.load(); }

// ---------------------------------------------------------------- evaluator source
struct Sym {
  std::string e;
  bool isInt;
};
std::string D(const Sym& s) { return s.isInt ? "((double)(" + s.e + "))" : s.e; }
std::string I(const Sym& s) { return s.isInt ? s.e : "((ws::i64)(" + s.e + "))"; }

struct ColUse {
  int t = 0;
  bool enc = false;   // the engine hints that some segments of this column are encoded
  bool vec = false;   // only used by vector functions (no row values loaded)
};

struct Gen {
  const ws_expr_env& env;
  int ncols;
  std::map<int, ColUse> cols;
  std::set<int> iconsts, dconsts;
  // common subexpressions of keys and aggregates: computed once per row into temporaries (prep)
  bool cse = false;
  std::map<std::string, std::string> tempOf;
  std::vector<std::pair<std::string, bool>> temps;  // (expression, is int) in dependency order

  Sym memo(const Sym& r) {
    if (!cse) return r;
    auto it = tempOf.find(r.e);
    if (it != tempOf.end()) return {it->second, r.isInt};
    const std::string name = "t" + std::to_string(temps.size()) + "[i]";
    tempOf.emplace(r.e, name);
    temps.emplace_back(r.e, r.isInt);
    return {name, r.isInt};
  }

  void useCol(int c, bool vecOnly) {
    auto it = cols.find(c);
    if (it == cols.end()) {
      ColUse u;
      u.t = env.cols[c].t;
      u.enc = env.cols[c].enc != 0;
      u.vec = vecOnly;
      cols.emplace(c, u);
    } else if (!vecOnly) {
      it->second.vec = false;
    }
  }
  std::string cv(int c) { return "c" + std::to_string(c) + "[i]"; }

  Sym node(const TypedProg& t, int ni) {
    const TNode& n = t.nodes[ni];
    const Sym r = node0(t, ni);
    if (n.op == WS_OP_COL || n.op == WS_OP_COLRAW || n.op == WS_OP_CONST) return r;
    return memo(r);
  }
  Sym node0(const TypedProg& t, int ni) {
    const TNode& n = t.nodes[ni];
    auto kid = [&](int k) { return node(t, n.kid[k]); };
    const std::string arg = std::to_string(n.arg);
    switch (n.op) {
      case WS_OP_COL: {
        useCol(n.arg, false);
        const int ty = env.cols[n.arg].t;
        const std::string v = cv(n.arg);
        if (ty == 0 || ty == 1) return {"((ws::i64)" + v + ")", true};
        if (ty == 2) return {v, false};
        if (ty == 3) return {"ws::nullIfI32(" + v + ")", false};
        if (ty == 4) return {"ws::nullIfI64(" + v + ")", false};
        if (ty == 6) {
          long long p = 1;
          for (int s = 0; s < env.cols[n.arg].scale; ++s) p *= 10;
          return {"ws::decOf(" + v + "," + std::to_string(p) + ".0)", false};
        }
        return {"ws::nanv()", false};
      }
      case WS_OP_COLRAW: {
        useCol(n.arg, false);
        if (n.isInt) return {"((ws::i64)" + cv(n.arg) + ")", true};
        return {"ws::nullIfI64(" + cv(n.arg) + ")", false};
      }
      case WS_OP_CONST:
        if (n.isInt) {
          iconsts.insert(n.arg);
          return {"ik" + arg + "()", true};
        }
        dconsts.insert(n.arg);
        return {"k" + arg + "()", false};
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL: {
        const Sym a = kid(0), b = kid(1);
        if (n.isInt)
          return {std::string(n.op == WS_OP_ADD ? "ws::iaddf(" : n.op == WS_OP_SUB ? "ws::isubf(" : "ws::imulf(") + a.e + "," + b.e + ",ofl)", true};
        const char* o = n.op == WS_OP_ADD ? "+" : n.op == WS_OP_SUB ? "-" : "*";
        return {"(" + D(a) + o + D(b) + ")", false};
      }
      case WS_OP_DIV: return {"ws::divz(" + D(kid(0)) + "," + D(kid(1)) + ")", false};
      case WS_OP_MOD: return {"fmod(" + D(kid(0)) + "," + D(kid(1)) + ")", false};
      case WS_OP_NEG: {
        const Sym a = kid(0);
        if (n.isInt) return {"((ws::i64)(0ull-(ws::u64)(" + a.e + ")))", true};
        return {"(-(" + a.e + "))", false};
      }
      case WS_OP_EQ: case WS_OP_NE: case WS_OP_LT: case WS_OP_LE: case WS_OP_GT: case WS_OP_GE: {
        static const char* ops[] = {"==", "!=", "<", "<=", ">", ">="};
        const Sym a = kid(0), b = kid(1);
        if (n.isInt) return {"((ws::i64)((" + a.e + ")" + ops[n.op - WS_OP_EQ] + "(" + b.e + ")))", true};
        return {"ws::cmp3(" + std::to_string(n.op - WS_OP_EQ) + "," + D(a) + "," + D(b) + ")", false};
      }
      case WS_OP_AND: case WS_OP_OR: {
        const Sym a = kid(0), b = kid(1);
        if (n.isInt)
          return {"((ws::i64)(((" + a.e + ")!=0)" + (n.op == WS_OP_AND ? "&&" : "||") + "((" + b.e + ")!=0)))", true};
        return {std::string(n.op == WS_OP_AND ? "ws::and3(" : "ws::or3(") + D(a) + "," + D(b) + ")", false};
      }
      case WS_OP_NOT: {
        const Sym a = kid(0);
        if (n.isInt) return {"((ws::i64)((" + a.e + ")==0))", true};
        return {"ws::not3(" + a.e + ")", false};
      }
      case WS_OP_INSET: {
        const Sym a = kid(0);
        if (n.isInt) return {"ws::insetI(L.env.sets[" + arg + "],L.env.setSize[" + arg + "]," + a.e + ")", true};
        return {"ws::insetD(L.env.sets[" + arg + "],L.env.setSize[" + arg + "]," + a.e + ")", false};
      }
      case WS_OP_SELECT: {
        const Sym c = kid(0), a = kid(1), b = kid(2);
        const std::string cond = c.isInt ? "((" + c.e + ")!=0)" : "ws::truthy(" + c.e + ")";
        if (n.isInt) return {"(" + cond + "?(" + a.e + "):(" + b.e + "))", true};
        return {"(" + cond + "?" + D(a) + ":" + D(b) + ")", false};
      }
      case WS_OP_YEAR: {
        const Sym a = kid(0);
        if (n.isInt) return {"ws::yearOf(" + a.e + ")", true};
        return {"ws::yearD(" + a.e + ")", false};
      }
      case WS_OP_ISNULL: {
        const Sym a = kid(0);
        if (a.isInt) return {"0ll", true};
        return {"((ws::i64)ws::isnul(" + a.e + "))", true};
      }
      case WS_OP_COALESCE: {
        const Sym a = kid(0), b = kid(1);
        if (a.isInt) return a;
        return {"ws::coalesce2(" + a.e + "," + D(b) + ")", false};
      }
      case WS_OP_NULLIF: return {"ws::nullif2(" + D(kid(0)) + "," + D(kid(1)) + ")", false};
      case WS_OP_CALL1: return {"ws::call1(" + arg + "," + D(kid(0)) + ")", false};
      case WS_OP_CALL2: return {"ws::call2(" + arg + "," + D(kid(0)) + "," + D(kid(1)) + ")", false};
      case WS_OP_DICTMAP:
        return {"ws::dictmapD(L.env.maps[" + arg + "],L.env.mapSize[" + arg + "]," + D(kid(0)) + ")", false};
      case WS_OP_INSORTED:
        return {"ws::insortedD(L.env.maps[" + arg + "],L.env.mapSize[" + arg + "]," + D(kid(0)) + ")", false};
      case WS_OP_VDOT: case WS_OP_VEUC: {
        const int slot = n.arg & 255, m = n.arg >> 8;
        useCol(slot, true);
        const std::string ms = std::to_string(m);
        return {std::string("ws::vecD(") + (n.op == WS_OP_VDOT ? "true" : "false") + ",(const float*)v" +
                    std::to_string(slot) + ".d,rb+i,L.env.maps[" + ms + "],L.env.mapSize[" + ms + "])",
                false};
      }
    }
    throw Error("codegen: unknown opcode", WS_ERR_INTERNAL);
  }
  Sym prog(ws_prog p) {
    const TypedProg t = typeProg(env, p, ncols);
    return node(t, t.root);
  }
};

const char* valType(const ColUse& u) {
  if (u.t == 2) return "double";
  if (u.t == 0 || u.t == 3) return "int";  // encoded int32 columns decode to int32 values too
  return "ws::i64";
}

}  // namespace

// Generated evaluator for one plan (see the evaluator contract in ws_kern.cuh).
std::string genEvaluator(const ws_expr_env& env, int ncols, const ws_agg_plan& plan, int fnKind, int* stageBytesOut) {
  Gen g{env, ncols, {}, {}, {}};
  const bool agg = fnKind == WS_JF_NOKEYS || fnKind == WS_JF_GROUPED || fnKind == WS_JF_DENSE;
  const Sym where = plan.hasWhere ? g.prog(plan.where) : Sym{"1", true};
  std::vector<Sym> keys, aggs;
  SlotLayout lay;
  if (agg) {
    lay = layoutOf(plan);
    g.cse = true;
    for (int k = 0; k < plan.nkeys; ++k) keys.push_back(g.prog(plan.keys[k]));
    for (int a = 0; a < plan.naggs; ++a) {
      if (plan.ops[a] == WS_AGG_COUNT || lay.kind[a] == SK_NONE) {
        aggs.push_back({"0", true});
        continue;
      }
      if (plan.aggNull[a]) {  // a nullable integer column read raw (its NULL sentinel is skipped)
        const ws_instr in = env.code[plan.aggs[a].start];
        if (plan.aggs[a].len != 1 || in.op != WS_OP_COL) throw Error("codegen: aggNull on a non-column", WS_ERR_INTERNAL);
        g.useCol(in.arg, false);
        aggs.push_back({"c" + std::to_string(in.arg) + "[i]", true});
        continue;
      }
      aggs.push_back(g.prog(plan.aggs[a]));
    }
    g.cse = false;
  }
  const int nk = agg ? plan.nkeys : 0, na = agg ? plan.naggs : 1;
  std::ostringstream o;
  o << "struct QEv {\n";
  // staged columns: every column whose row values are loaded; stage slot = the type's widest storage
  std::vector<int> staged;
  std::vector<int> soff;
  int stageBytes = 0;
  for (auto& [c, u] : g.cols) {
    if (u.vec) continue;
    staged.push_back(c);
    soff.push_back(stageBytes);
    stageBytes += ((u.t == 0 || u.t == 3) ? 4 : 8) * 1024;  // kTile rows
  }
  if (stageBytesOut) *stageBytesOut = stageBytes;
  o << "  static constexpr int NK = " << std::max(nk, 1) << ", NA = " << na << ", RW = " << (agg ? lay.rw : 1)
    << ", FRW = " << std::max(agg ? lay.frw : 1, 1) << ";\n";
  o << "  static constexpr bool STAGED = " << (staged.empty() ? "false" : "true") << ";\n";
  // resident CTAs of the direct-load private-row kernel (a register budget of 85 per thread)
  static const int privMinBlocks = [] {
    const char* e = getenv("WARPSTORE_B200_PRIV_MIN_BLOCKS");
    const int v = e ? atoi(e) : 0;
    return v >= 1 && v <= 4 ? v : 2;
  }();
  o << "  static constexpr int PRIV_MIN_BLOCKS = " << privMinBlocks << ";\n";
  o << "  static constexpr int HASH_MULTI_MIN_BLOCKS = 3;\n";  // the multi-query hash scan's register bound
  o << "  static constexpr int NSC = " << std::max<size_t>(staged.size(), 1) << ", STAGE_BYTES = " << stageBytes << ";\n";
  o << "  struct Stage { const unsigned char* d[NSC]; int w[NSC]; unsigned bytes; int ok; };\n";
  o << "  __device__ static void stageBind(const ws::Launch& l, int b, Stage& st) {\n";
  o << "    const ws_col_view* cv = l.cols + (ws::i64)b * l.ncols;\n    st.bytes = 0; st.ok = 1;\n";
  for (size_t j = 0; j < staged.size(); ++j)
    o << "    { const ws::ColRef v = ws::resolveCol(cv[" << staged[j] << "]); st.d[" << j << "] = v.d; st.w[" << j
      << "] = v.width; st.bytes += ws::kTile * v.width; st.ok &= (((unsigned long long)v.d & 15) == 0) && v.width > 0; }\n";
  o << "  }\n";
  o << "  __device__ static void stageIssue(const Stage& st, ws::i64 tr0, unsigned dst, unsigned bar) {\n";
  for (size_t j = 0; j < staged.size(); ++j)
    o << "    ws::bulkG2S(dst + " << soff[j] << ", st.d[" << j << "] + tr0 * st.w[" << j << "], ws::kTile * st.w[" << j
      << "], bar);\n";
  o << "  }\n";
  // ofl: overflow of this thread's checked integer arithmetic (rows that passed or were filtered),
  // stored to the plan's flag once by finish()
  o << "  const ws::Launch& L;\n  mutable unsigned ofl;\n  bool fastOk;\n  ws::i64 rb;\n";
  o << "  const ws_col_view* cvb;  // the bound batch's views (bit-packed / run-length columns decode from them)\n";
  // plan constants are read from the launch descriptor (constant bank) where used, not kept in registers
  for (int k : g.iconsts)
    o << "  __device__ __forceinline__ ws::i64 ik" << k << "() const { return __double_as_longlong(L.env.consts[" << k << "]); }\n";
  for (int k : g.dconsts) o << "  __device__ __forceinline__ double k" << k << "() const { return L.env.consts[" << k << "]; }\n";
  for (size_t j = 0; j < g.temps.size(); ++j) o << "  " << (g.temps[j].second ? "ws::i64" : "double") << " t" << j << "[4];\n";
  for (auto& [c, u] : g.cols) {
    o << "  ws::ColRef v" << c << ";\n";
    if (!u.vec) o << "  " << valType(u) << " c" << c << "[4];\n";
  }
  o << "  __device__ QEv(const ws::Launch& l) : L(l), ofl(0), fastOk(false), rb(0), cvb(nullptr) {}\n";
  o << "  __device__ __forceinline__ int nk() const { return " << nk << "; }\n";
  o << "  __device__ __forceinline__ int na() const { return " << na << "; }\n";
  o << "  __device__ __forceinline__ int rowWords() const { return " << (agg ? lay.rw : 1) << "; }\n";
  o << "  __device__ __forceinline__ int kind(int a) const { switch (a) {";
  if (agg)
    for (int a = 0; a < na; ++a) o << " case " << a << ": return " << (int)lay.kind[a] << ";";
  o << " } return 0; }\n";
  o << "  __device__ __forceinline__ int woff(int a) const { switch (a) {";
  if (agg)
    for (int a = 0; a < na; ++a) o << " case " << a << ": return " << lay.woff[a] << ";";
  o << " } return 0; }\n";
  o << "  __device__ __forceinline__ int fastWords() const { return " << std::max(agg ? lay.frw : 1, 1) << "; }\n";
  o << "  __device__ __forceinline__ int fwoff(int a) const { switch (a) {";
  if (agg)
    for (int a = 0; a < na; ++a) o << " case " << a << ": return " << lay.fwoff[a] << ";";
  o << " } return 0; }\n";
  o << "  __device__ __forceinline__ bool keyInt(int k) const { switch (k) {";
  for (int k = 0; k < nk; ++k) o << " case " << k << ": return " << (plan.keyInt[k] ? "true" : "false") << ";";
  o << " } return false; }\n";
  // batch binding: resolve the views of the columns used, check vector-load alignment
  o << "  __device__ __forceinline__ void bind(const ws::Launch& l, int b) {\n";
  o << "    const ws_col_view* cv = l.cols + (ws::i64)b * l.ncols;\n    cvb = cv;\n";
  std::string fast = "true";
  for (auto& [c, u] : g.cols) {
    o << "    v" << c << " = ws::resolveCol(cv[" << c << "]);\n";
    if (!u.vec) fast += " && ws::aligned4(v" + std::to_string(c) + ")";
  }
  o << "    fastOk = " << fast << ";\n  }\n";
  // loads of 4 consecutive rows: one branch between the all-vector form (whole aligned groups) and the
  // element-wise form (ragged last group, unaligned views)
  auto emitLoads = [&](const char* fast) {
    for (auto& [c, u] : g.cols) {
      if (u.vec) continue;
      const std::string C = std::to_string(c), v = "v" + C, a = "c" + C, F = std::string(",") + fast + ",nv)";
      if (u.t == 2) {
        if (u.enc)
          o << "      if (" << v << ".enc) ws::load4encD(" << a << "," << v << ".d + r0 * " << v << ".width," << v << ".dict," << v
            << ".enc," << v << ".base," << v << ".p10" << F << "; else ";
        o << "      ws::load4f64(" << a << ",(const double*)" << v << ".d + r0" << F << ";\n";
      } else if (u.t == 0 || u.t == 3) {
        if (u.enc)
          o << "      if (" << v << ".enc >= 7) { ws::i64 u_[4]; ws::load4encView(u_,cvb + " << C
            << ",r0,(ws::i64)WS_NULL_I32,nv); for (int j = 0; j < 4; ++j) " << a << "[j] = (int)u_[j]; } else if ("
            << v << ".enc) { ws::i64 t_[4]; ws::load4enc(t_," << v << ".d + r0 * " << v << ".width," << v
            << ".enc," << v << ".base,(ws::i64)WS_NULL_I32" << F << "; for (int j = 0; j < 4; ++j) " << a
            << "[j] = (int)t_[j]; } else ";
        o << "      ws::load4i32(" << a << ",(const int*)" << v << ".d + r0" << F << ";\n";
      } else {
        if (u.enc)
          o << "      if (" << v << ".enc >= 7) { ws::i64 u_[4]; ws::load4encView(u_,cvb + " << C
            << ",r0,(ws::i64)WS_NULL_I64,nv); for (int j = 0; j < 4; ++j) " << a << "[j] = u_[j]; }"
            << " else if (" << v << ".enc) ws::load4enc(" << a << "," << v << ".d + r0 * " << v << ".width," << v << ".enc,"
            << v << ".base,(ws::i64)WS_NULL_I64" << F << "; else ";
        o << "      ws::load4i64(" << a << ",(const ws::i64*)" << v << ".d + r0" << F << ";\n";
      }
    }
  };
  o << "  __device__ __forceinline__ void load(ws::i64 r0, bool fast, int nv) {\n    rb = r0;\n    if (fast) {\n";
  emitLoads("true");
  o << "    } else {\n";
  emitLoads("false");
  o << "    }\n  }\n";
  // the same rows from a shared-memory stage (whole tile; rt = the thread's first row in it)
  o << "  __device__ __forceinline__ void loadStage(const unsigned char* st, int rt) {\n";
  for (size_t j = 0; j < staged.size(); ++j) {
    const int c = staged[j];
    const ColUse& u = g.cols[c];
    const std::string C = std::to_string(c), v = "v" + C, a = "c" + C;
    const std::string src = "st + " + std::to_string(soff[j]) + " + rt * " + v + ".width";
    if (u.t == 2) {
      if (u.enc) o << "    if (" << v << ".enc) ws::stage4encD(" << a << "," << src << "," << v << ".dict," << v << ".enc," << v << ".base," << v << ".p10); else ";
      o << "    ws::stage4f64(" << a << "," << src << ");\n";
    } else if (u.t == 0 || u.t == 3) {
      if (u.enc)
        o << "    if (" << v << ".enc) { ws::i64 t_[4]; ws::stage4enc(t_," << src << "," << v << ".enc," << v
          << ".base,(ws::i64)WS_NULL_I32); for (int j = 0; j < 4; ++j) " << a << "[j] = (int)t_[j]; } else ws::stage4i32(" << a
          << "," << src << ");\n";
      else o << "    ws::stage4i32(" << a << "," << src << ");\n";
    } else {
      if (u.enc) o << "    if (" << v << ".enc) ws::stage4enc(" << a << "," << src << "," << v << ".enc," << v << ".base,(ws::i64)WS_NULL_I64); else ";
      o << "    ws::stage4i64(" << a << "," << src << ");\n";
    }
  }
  o << "  }\n";
  // per-row common subexpressions (rows that did not pass the filter compute unused values and
  // raise no overflow flag)
  // Integer products among the temporaries are first computed as 32 x 32-bit products (exact when every
  // operand fits in int32, no branch); a row with a wider operand recomputes them with tested products.
  o << "  __device__ __forceinline__ void prep(int i, bool live) {\n";
  if (!g.temps.empty()) o << "    unsigned ofl = 0;\n";
  const std::string mulHead = "ws::imulf(", mulTail = ",ofl)";
  bool anyMul = false;
  for (auto& t : g.temps)
    anyMul |= t.first.compare(0, mulHead.size(), mulHead) == 0 && t.first.size() > mulTail.size() &&
              t.first.compare(t.first.size() - mulTail.size(), mulTail.size(), mulTail) == 0;
  if (anyMul) {
    o << "    unsigned wide = 0;\n";
    for (size_t j = 0; j < g.temps.size(); ++j) {
      const std::string& e = g.temps[j].first;
      const bool mul = e.compare(0, mulHead.size(), mulHead) == 0 && e.size() > mulTail.size() &&
                       e.compare(e.size() - mulTail.size(), mulTail.size(), mulTail) == 0;
      o << "    t" << j << "[i] = "
        << (mul ? "ws::imul32w(" + e.substr(mulHead.size(), e.size() - mulHead.size() - mulTail.size()) + ",wide)" : e)
        << ";\n";
    }
    o << "    if (wide) {\n      ofl = 0;\n";
    for (size_t j = 0; j < g.temps.size(); ++j) o << "      t" << j << "[i] = " << g.temps[j].first << ";\n";
    o << "    }\n";
  } else {
    for (size_t j = 0; j < g.temps.size(); ++j) o << "    t" << j << "[i] = " << g.temps[j].first << ";\n";
  }
  if (!g.temps.empty()) o << "    this->ofl |= live ? ofl : 0u;\n";
  o << "  }\n";
  o << "  __device__ __forceinline__ void finish() const { if (ofl) *L.env.ovf = 1; }\n";
  o << "  __device__ __forceinline__ bool where(int i) const { return "
    << (where.isInt ? "(" + where.e + ") != 0" : "ws::truthy(" + where.e + ")") << "; }\n";
  o << "  __device__ __forceinline__ ws::i64 ikey(int k, int i) const { switch (k) {";
  for (int k = 0; k < nk; ++k) o << "\n    case " << k << ": return " << I(keys[k]) << ";";
  o << " } return 0; }\n";
  o << "  __device__ __forceinline__ double dkey(int k, int i) const { switch (k) {";
  for (int k = 0; k < nk; ++k) o << "\n    case " << k << ": return " << D(keys[k]) << ";";
  o << " } return 0; }\n";
  o << "  __device__ __forceinline__ bool ival(int a, int i, ws::i64& v) const { switch (a) {";
  if (agg)
    for (int a = 0; a < na; ++a) {
      if (plan.ops[a] == WS_AGG_COUNT || lay.kind[a] == SK_NONE) continue;
      if (!(lay.kind[a] == SK_ISUM || lay.kind[a] == SK_IMIN || lay.kind[a] == SK_IMAX)) continue;
      if (plan.aggNull[a])
        o << "\n    case " << a << ": v = " << aggs[a].e << "; return v != "
          << (plan.aggNull[a] == 3 ? "(ws::i64)WS_NULL_I32" : "(ws::i64)WS_NULL_I64") << ";";
      else
        o << "\n    case " << a << ": v = " << I(aggs[a]) << "; return true;";
    }
  o << " } v = 0; return false; }\n";
  o << "  __device__ __forceinline__ double dval(int a, int i) const { switch (a) {";
  if (agg)
    for (int a = 0; a < na; ++a) {
      if (!(lay.kind[a] == SK_DSUM || lay.kind[a] == SK_DMIN || lay.kind[a] == SK_DMAX)) continue;
      o << "\n    case " << a << ": return " << D(aggs[a]) << ";";
    }
  o << " } return 0; }\n";
  o << "};\n";
  return o.str();
}

namespace {

// kernels each plan kind compiles (prefix wsq)
const char* kindKernels(int fnKind) {
  switch (fnKind) {
    case WS_JF_NOKEYS: return "WS_K_NOKEYS(QEv, wsq)\nWS_K_MULTI_NOKEYS(QEv, wsq)\n";
    case WS_JF_GROUPED: return "WS_K_HASH(QEv, wsq)\nWS_K_MULTI_HASH(QEv, wsq)\n";
    case WS_JF_DENSE:
      return "WS_K_DENSE_PRIV(QEv, wsq)\nWS_K_DENSE_SHARED(QEv, wsq)\nWS_K_DENSE_GLOBAL(QEv, wsq)\n"
             "WS_K_MULTI_DENSE_PRIV(QEv, wsq)\n";
    default: return "WS_K_SELECT_COUNT(QEv, wsq)\nWS_K_SELECT_WRITE(QEv, wsq)\n";
  }
}

uint64_t fnv64(const std::string& s, uint64_t h) {
  for (unsigned char c : s) h = (h ^ c) * 0x100000001b3ull;
  return h;
}

struct Build {
  std::string src, key, path;
  std::vector<std::string> opts;
};

std::vector<std::string> archOpts(int a) {
  return {std::string("--gpu-architecture=sm_") + std::to_string(a) + (a == 100 || a == 90 ? "a" : ""), "--std=c++17",
          "--generate-line-info", "-DNDEBUG"};
}

// NVRTC compile of a module body to a cubin (no device needed); throws with the log on failure.
std::string nvrtcCubin(const std::string& src, const std::vector<std::string>& optsIn) {
  nvrtcProgram prog;
  const char* hdrs[] = {kWsTypesSrc, kWsDevSrc, kWsKernSrc};
  const char* names[] = {"ws_types.h", "ws_dev.cuh", "ws_kern.cuh"};
  if (nvrtcCreateProgram(&prog, src.c_str(), "ws_query.cu", 3, hdrs, names) != NVRTC_SUCCESS)
    throw Error("codegen: nvrtcCreateProgram failed", WS_ERR_INTERNAL);
  // WARPSTORE_B200_JIT_VERBOSE=1: print the compiler's resource report (registers, spills) per kernel
  static const bool verbose = getenv("WARPSTORE_B200_JIT_VERBOSE") && atoi(getenv("WARPSTORE_B200_JIT_VERBOSE")) > 0;
  std::vector<const char*> opts;
  for (auto& o : optsIn) opts.push_back(o.c_str());
  if (verbose) opts.push_back("--ptxas-options=-v");
  const nvrtcResult rc = nvrtcCompileProgram(prog, (int)opts.size(), opts.data());
  if (verbose && rc == NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    nvrtcGetProgramLog(prog, log.data());
    int maj = 0, mnr = 0;
    nvrtcVersion(&maj, &mnr);
    fprintf(stderr, "[warpstore_b200 jit] NVRTC %d.%d\n%s\n", maj, mnr, log.c_str());
  }
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    nvrtcGetProgramLog(prog, log.data());
    nvrtcDestroyProgram(&prog);
    throw Error("codegen: NVRTC failed: " + log, WS_ERR_INTERNAL);
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  std::string image(n, '\0');
  nvrtcGetCUBIN(prog, image.data());
  nvrtcDestroyProgram(&prog);
  return image;
}

Build planBuild(const std::string& body) {
  Build b;
  b.src = "#include \"ws_kern.cuh\"\n" + body;
  const int a = arch();
  b.opts = archOpts(a);
  if (!gDiskDir.empty()) {
    int maj = 0, min = 0;
    nvrtcVersion(&maj, &min);
    b.key = "nvrtc " + std::to_string(maj) + "." + std::to_string(min) + "\n";
    for (auto& o : b.opts) b.key += o + "\n";
    b.key += std::string(kWsTypesSrc) + kWsDevSrc + kWsKernSrc + b.src;
    char name[48];
    snprintf(name, sizeof name, "%016llx%016llx.wsplan", (unsigned long long)fnv64(b.key, 0xcbf29ce484222325ull),
             (unsigned long long)fnv64(b.key, 0x84222325cbf29ce4ull));
    b.path = gDiskDir + "/" + name;
  }
  return b;
}

// Plan file: "WSPLAN01", key length, key, image length, image, FNV-64 of the image.
bool diskLoad(const Build& b, std::string& image) {
  if (b.path.empty()) return false;
  std::ifstream f(b.path, std::ios::binary);
  if (!f) return false;
  char magic[8];
  uint64_t kl = 0, il = 0, sum = 0;
  f.read(magic, 8);
  f.read((char*)&kl, 8);
  if (!f || memcmp(magic, "WSPLAN01", 8) != 0 || kl != b.key.size()) return false;
  std::string k(kl, '\0');
  f.read(k.data(), (std::streamsize)kl);
  f.read((char*)&il, 8);
  if (!f || k != b.key || il > (1ull << 30)) return false;
  image.assign(il, '\0');
  f.read(image.data(), (std::streamsize)il);
  f.read((char*)&sum, 8);
  if (!f || sum != fnv64(image, 0xcbf29ce484222325ull)) {
    fprintf(stderr, "[warpstore_b200] plan cache file %s is corrupt; recompiling\n", b.path.c_str());
    return false;
  }
  return true;
}

void diskStore(const Build& b, const std::string& image) {
  if (b.path.empty()) return;
  const std::string tmp = b.path + ".tmp" + std::to_string(std::hash<std::thread::id>{}(std::this_thread::get_id()));
  {
    std::ofstream f(tmp, std::ios::binary);
    const uint64_t kl = b.key.size(), il = image.size(), sum = fnv64(image, 0xcbf29ce484222325ull);
    f.write("WSPLAN01", 8);
    f.write((const char*)&kl, 8);
    f.write(b.key.data(), (std::streamsize)kl);
    f.write((const char*)&il, 8);
    f.write(image.data(), (std::streamsize)il);
    f.write((const char*)&sum, 8);
    if (!f) return;
  }
  std::error_code ec;
  std::filesystem::rename(tmp, b.path, ec);
}

// Compiles (or loads from disk) the module of `body`; throws on failure.
CUmodule compileModule(const std::string& body, bool* fromDisk) {
  ensureInit();
  Build b = planBuild(body);
  std::string image;
  bool disk = diskLoad(b, image);
  if (!disk) {
    image = nvrtcCubin(b.src, b.opts);
    diskStore(b, image);
  }
  if (fromDisk) *fromDisk = disk;
  cudaFree(nullptr);  // make sure this thread has the primary context current
  CUmodule mod;
  WS_CKD(drv().moduleLoadData(&mod, image.data()));
  return mod;
}

void compileProgram(ws_jit_program& p) {
  const std::string body = p.source + kindKernels(p.fnKind);
  bool disk = false;
  p.module = compileModule(body, &disk);
  p.fromDisk = disk;
  static const char* names[K_COUNT_] = {"wsq_nokeys", "wsq_dense_shared", "wsq_dense_global", "wsq_hash",
                                        "wsq_select_count", "wsq_select_write", "wsq_dense_priv",
                                        "wsq_dense_priv_staged", "wsq_multi_nokeys", "wsq_multi_dense_priv",
                                        "wsq_multi_hash"};
  for (int k = 0; k < K_COUNT_; ++k) {
    CUfunction f = nullptr;
    if (drv().moduleGetFunction(&f, p.module, names[k]) == CUDA_SUCCESS) p.kernels.fn[k] = f;
  }
  p.kernels.interp = false;
}

void compileAndPublish(const std::shared_ptr<ws_jit_program>& p) {
  auto t0 = std::chrono::steady_clock::now();
  bool ok = false;
  try {
    compileProgram(*p);
    ok = true;
  } catch (const std::exception& e) {
    fprintf(stderr, "[warpstore_b200] codegen failed, using the interpreter: %s\n", e.what());
  }
  p->compileMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  p->state.store(ok ? 1 : 2, std::memory_order_release);
}

}  // namespace

}  // namespace ws

using namespace ws;

extern "C" {

int ws_jit_set_mode(int mode) {
  tMode = mode;
  return WS_OK;
}
int ws_jit_mode(void) { return jitMode(); }
int ws_jit_set_default_mode(int mode) {
  gDefaultMode = mode;
  return WS_OK;
}
int ws_jit_set_cache_dir(const char* dir) {
  return guardedCall([&] {
    std::lock_guard<std::mutex> g(gMu);
    if (!dir || !*dir) {
      gDiskDir.clear();
      tuneSetDir("");
      return;
    }
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    gDiskDir = ec ? "" : dir;
    if (ec) throw Error(std::string("plan cache directory unusable: ") + ec.message(), WS_ERR_ARG);
    tuneSetDir(gDiskDir);  // launch shapes tuned earlier for these plans
  });
}

int ws_prog_is_int(const ws_expr_env* env, ws_prog p) {
  int r = 0;
  guardedCall([&] { r = typeProg(*env, p, WS_MAX_COLS).isInt() ? 1 : 0; });
  return r;
}

int ws_jit_get(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, const char* kind,
               const ws_jit_program** out) {
  return guardedCall([&] {
    *out = nullptr;
    const int mode = jitMode();
    if (mode == WS_JIT_OFF) return;
    int stageBytes = 0;
    const std::string ev = genEvaluator(*env, ncols, *plan, fn, &stageBytes);
    const std::string key = std::to_string(fn) + "\n" + ev;
    std::shared_ptr<ws_jit_program> p;
    bool fresh = false;
    {
      std::lock_guard<std::mutex> g(gMu);
      auto it = gCache.find(key);
      if (it != gCache.end()) {
        p = it->second;
      } else {
        p = std::make_shared<ws_jit_program>();
        p->id = (int)gById.size() + 1;
        p->fnKind = fn;
        p->kind = kind ? kind : "";
        p->sql = tSql;
        p->source = ev;
        p->stageBytes = stageBytes;
        gById.push_back(p);
        gCache.emplace(key, p);
        fresh = true;
      }
    }
    if (fresh) {
      if (mode == WS_JIT_SYNC) {
        compileAndPublish(p);
        if (p->state.load() == 1) {
          if (p->fromDisk) ++tInfo.from_disk;
          else ++tInfo.compiled;
          tInfo.compile_ms += p->compileMs;
        }
      } else {
        std::thread([p] { compileAndPublish(p); }).detach();  // run interpreted now, compiled next time
      }
    } else if (mode == WS_JIT_SYNC) {
      for (int spins = 0; p->state.load(std::memory_order_acquire) == 0; ++spins)  // compiled by another thread
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
    const int st = p->state.load(std::memory_order_acquire);
    if (st != 1) {
      if (st == 0) ++tInfo.background;
      return;
    }
    if (!fresh) ++tInfo.hits;
    std::lock_guard<std::mutex> g(gMu);
    if (std::find(tUsed.begin(), tUsed.end(), p.get()) == tUsed.end()) tUsed.push_back(p.get());
    *out = p.get();
  });
}

int ws_codegen_source(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, char* buf, size_t size,
                      size_t* needed) {
  return guardedCall([&] {
    const std::string ev = genEvaluator(*env, ncols, *plan, fn, nullptr);
    if (needed) *needed = ev.size() + 1;
    if (buf && size) {
      const size_t n = std::min(size - 1, ev.size());
      memcpy(buf, ev.data(), n);
      buf[n] = 0;
    }
  });
}

int ws_codegen_compile_check(const ws_expr_env* env, int ncols, const ws_agg_plan* plan, int fn, int arch_sm,
                             size_t* cubin_bytes) {
  return guardedCall([&] {
    const std::string body = genEvaluator(*env, ncols, *plan, fn, nullptr) + kindKernels(fn);
    const std::string image = nvrtcCubin("#include \"ws_kern.cuh\"\n" + body, archOpts(arch_sm));
    if (cubin_bytes) *cubin_bytes = image.size();
  });
}

int ws_jit_program_info(const ws_jit_program* p, ws_jit_info* info) {
  if (!p || !info) return WS_ERR_ARG;
  info->id = p->id;
  info->fn_kind = p->fnKind;
  info->state = p->state.load();
  info->from_disk = p->fromDisk;
  info->compile_ms = p->compileMs;
  info->execs = p->execs;
  info->total_ms = p->totalMs;
  info->last_ms = p->lastMs;
  info->source_bytes = (int64_t)p->source.size();
  return WS_OK;
}

int ws_jit_source_of(int id, char* buf, size_t size, size_t* needed) {
  std::lock_guard<std::mutex> g(gMu);
  for (auto& p : gById)
    if (p->id == id) {
      if (needed) *needed = p->source.size() + 1;
      if (buf && size) {
        const size_t n = std::min(size - 1, p->source.size());
        memcpy(buf, p->source.data(), n);
        buf[n] = 0;
      }
      return WS_OK;
    }
  if (needed) *needed = 0;
  return WS_ERR_ARG;
}

int ws_jit_plan_text(int id, int field, char* buf, size_t size, size_t* needed) {
  if (field < 0 || field > 2) return WS_ERR_ARG;
  std::lock_guard<std::mutex> g(gMu);
  for (auto& p : gById)
    if (p->id == id) {
      const std::string& t = field == 0 ? p->kind : field == 1 ? p->sql : p->source;
      if (needed) *needed = t.size() + 1;
      if (buf && size) {
        const size_t n = std::min(size - 1, t.size());
        memcpy(buf, t.data(), n);
        buf[n] = 0;
      }
      return WS_OK;
    }
  if (needed) *needed = 0;
  return WS_ERR_ARG;
}

int ws_jit_last_query_plans(int* ids, int max_ids, int* n) {
  *n = (int)tLastIds.size();
  for (int i = 0; i < *n && i < max_ids; ++i) ids[i] = tLastIds[(size_t)i];
  return *n > max_ids ? WS_ERR_SIZE : WS_OK;
}

int ws_jit_plan_cache_count(void) {
  std::lock_guard<std::mutex> g(gMu);
  return (int)gById.size();
}
int ws_jit_plan_cache_row(int i, ws_jit_info* info) {
  std::shared_ptr<ws_jit_program> p;
  {
    std::lock_guard<std::mutex> g(gMu);
    if (i < 0 || i >= (int)gById.size()) return WS_ERR_ARG;
    p = gById[i];
  }
  return ws_jit_program_info(p.get(), info);
}
int ws_jit_clear_cache(void) {
  // Modules stay loaded: a query on another thread may still be running one.
  std::lock_guard<std::mutex> g(gMu);
  gById.clear();
  gCache.clear();
  return WS_OK;
}
int ws_jit_begin_query(const char* sql) {
  tSql.clear();
  for (const char* c = sql ? sql : ""; *c; ++c) {
    const bool sp = *c == ' ' || *c == '\n' || *c == '\t' || *c == '\r';
    if (sp && (tSql.empty() || tSql.back() == ' ')) continue;
    tSql += sp ? ' ' : *c;
  }
  while (!tSql.empty() && tSql.back() == ' ') tSql.pop_back();
  tUsed.clear();
  tInfo = ws_jit_query_info{};
  return WS_OK;
}
int ws_jit_end_query(double query_ms, ws_jit_query_info* info) {
  std::lock_guard<std::mutex> g(gMu);
  tLastIds.clear();
  for (ws_jit_program* p : tUsed) tLastIds.push_back(p->id);
  for (ws_jit_program* p : tUsed) {
    ++p->execs;
    p->totalMs += query_ms;
    p->lastMs = query_ms;
  }
  tUsed.clear();
  if (info) *info = tInfo;
  return WS_OK;
}

}  // extern "C"
