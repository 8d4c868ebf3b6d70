// Plan analysis: expression typing, accumulator layout and interpreter code.
//
// Typing follows the reference's code generator (src/jit.cu:113-273) so that a query computes the same
// values here as under the engine's compiled plans: integer columns (I32 / I64), integer literals and
// arithmetic / comparisons / logic over integers stay int64 (checked for overflow); nullable integer
// columns, DECIMAL columns, doubles and every function are double-typed with NULL = NaN.
#include <cstring>

#include "ws_internal.h"

namespace ws {

TypedProg typeProg(const ws_expr_env& env, ws_prog p, int ncols) {
  TypedProg t;
  std::vector<int> st;
  auto pop = [&]() {
    if (st.empty()) throw Error("codegen: malformed expression", WS_ERR_INTERNAL);
    const int v = st.back();
    st.pop_back();
    return v;
  };
  if (p.len <= 0 || p.start < 0 || p.start + p.len > WS_MAX_CODE) throw Error("codegen: bad program range", WS_ERR_INTERNAL);
  for (int pc = p.start; pc < p.start + p.len; ++pc) {
    const ws_instr in = env.code[pc];
    TNode n;
    n.op = in.op;
    n.instrInt = in.isInt;
    n.arg = in.arg;
    auto kidsInt = [&](int a, int b) { return t.nodes[a].isInt && t.nodes[b].isInt; };
    switch (in.op) {
      case WS_OP_COL: {
        if (in.arg >= ncols) throw Error("codegen: column slot out of range", WS_ERR_INTERNAL);
        const int ty = env.cols[in.arg].t;
        n.isInt = ty == 0 || ty == 1;
        break;
      }
      case WS_OP_COLRAW:
        if (in.arg >= ncols) throw Error("codegen: column slot out of range", WS_ERR_INTERNAL);
        n.isInt = !(env.cols[in.arg].t == 6 && !in.isInt);
        break;
      case WS_OP_CONST:
        if (in.arg >= WS_MAX_CONSTS) throw Error("codegen: constant out of range", WS_ERR_INTERNAL);
        n.isInt = in.isInt != 0;
        break;
      case WS_OP_ADD: case WS_OP_SUB: case WS_OP_MUL: case WS_OP_EQ: case WS_OP_NE: case WS_OP_LT: case WS_OP_LE:
      case WS_OP_GT: case WS_OP_GE: case WS_OP_AND: case WS_OP_OR:
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = kidsInt(n.kid[0], n.kid[1]);
        break;
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
      case WS_OP_NEG: case WS_OP_NOT: case WS_OP_YEAR:
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[0]].isInt;
        break;
      case WS_OP_INSET:
        if (in.arg >= WS_MAX_SETS) throw Error("codegen: set out of range", WS_ERR_INTERNAL);
        n.kid[0] = pop();
        n.isInt = t.nodes[n.kid[0]].isInt;
        break;
      case WS_OP_ISNULL:
        n.kid[0] = pop();
        n.isInt = true;
        break;
      case WS_OP_CALL1:
        n.kid[0] = pop();
        n.isInt = false;
        break;
      case WS_OP_DICTMAP: case WS_OP_INSORTED:
        if (in.arg >= WS_MAX_SETS) throw Error("codegen: map out of range", WS_ERR_INTERNAL);
        n.kid[0] = pop();
        n.isInt = false;
        break;
      case WS_OP_SELECT:
        n.kid[2] = pop();
        n.kid[1] = pop();
        n.kid[0] = pop();
        n.isInt = kidsInt(n.kid[1], n.kid[2]);
        break;
      case WS_OP_VDOT: case WS_OP_VEUC:
        if ((in.arg & 255) >= ncols || (in.arg >> 8) >= WS_MAX_SETS) throw Error("codegen: vector operand out of range", WS_ERR_INTERNAL);
        n.isInt = false;
        break;
      default: throw Error("codegen: unknown opcode " + std::to_string(in.op), WS_ERR_INTERNAL);
    }
    t.nodes.push_back(n);
    st.push_back((int)t.nodes.size() - 1);
    if ((int)st.size() > WS_MAX_STACK) throw Error("codegen: expression too deeply nested", WS_ERR_INTERNAL);
  }
  if (st.size() != 1) throw Error("codegen: malformed expression", WS_ERR_INTERNAL);
  t.root = st[0];
  return t;
}

// Slot kinds (src/kernels.cuh:35-82 for the reference's accumulation rules): COUNT; integer SUM
// exact in 128 bits; integer MIN / MAX in int64; double SUM / MIN / MAX skipping NULL.  The high half
// of a split BIGINT SUM (aggPart 2) needs no accumulation of its own: the low slot holds the exact
// whole sum and both halves are produced from it.
SlotLayout layoutOf(const ws_agg_plan& plan) {
  SlotLayout L;
  if (plan.naggs < 1 || plan.naggs > WS_MAX_AGGS) throw Error("plan: bad aggregate count", WS_ERR_INTERNAL);
  if (plan.nkeys < 0 || plan.nkeys > WS_MAX_KEYS) throw Error("plan: bad key count", WS_ERR_INTERNAL);
  L.na = plan.naggs;
  int w = 1;
  for (int a = 0; a < plan.naggs; ++a) {
    const uint8_t op = plan.ops[a];
    uint8_t k;
    L.partner[a] = a;
    if (op == WS_AGG_COUNT) k = SK_COUNT;
    else if (op == WS_AGG_SUM && plan.aggPart[a] == 2 && a > 0 && plan.aggPart[a - 1] == 1 &&
             plan.ops[a - 1] == WS_AGG_SUM && plan.aggInt[a] && plan.aggInt[a - 1]) {
      // the engine allocates the high-half slot right after the low-half slot of the same column
      // (src/engine_select.cpp:707-715)
      k = SK_NONE;
      L.partner[a] = a - 1;
    } else if (op == WS_AGG_SUM) k = plan.aggInt[a] ? SK_ISUM : SK_DSUM;
    else if (op == WS_AGG_MIN) k = plan.aggInt[a] ? SK_IMIN : SK_DMIN;
    else if (op == WS_AGG_MAX) k = plan.aggInt[a] ? SK_IMAX : SK_DMAX;
    else throw Error("plan: unknown aggregate op", WS_ERR_INTERNAL);
    L.kind[a] = k;
    L.woff[a] = w;
    L.fwoff[a] = L.frw;
    w += k == SK_NONE ? 0 : k == SK_ISUM ? 2 : 1;
    L.frw += k == SK_NONE ? 0 : 1;
  }
  L.rw = w;
  return L;
}

static void emitTyped(const TypedProg& t, int ni, std::vector<TInstr>& out) {
  const TNode& n = t.nodes[ni];
  for (int k = 0; k < 3; ++k)
    if (n.kid[k] >= 0) emitTyped(t, n.kid[k], out);
  TInstr x{};
  x.op = n.op;
  x.rInt = n.isInt;
  x.aInt = n.kid[0] >= 0 ? t.nodes[n.kid[0]].isInt : 0;
  x.bInt = n.kid[1] >= 0 ? t.nodes[n.kid[1]].isInt : 0;
  x.cInt = n.kid[2] >= 0 ? t.nodes[n.kid[2]].isInt : 0;
  x.arg = n.arg;
  out.push_back(x);
}

void buildTProgs(const ws_expr_env& env, int ncols, const ws_agg_plan& plan, bool hasWhere, TProgs& out) {
  memset(&out, 0, sizeof out);
  std::vector<TInstr> code;
  auto add = [&](ws_prog p, int (&dst)[2]) {
    const TypedProg t = typeProg(env, p, ncols);
    dst[0] = (int)code.size();
    emitTyped(t, t.root, code);
    dst[1] = (int)code.size() - dst[0];
  };
  if (hasWhere) add(plan.where, out.where);
  for (int k = 0; k < plan.nkeys; ++k) add(plan.keys[k], out.keys[k]);
  const SlotLayout lay = layoutOf(plan);
  for (int a = 0; a < plan.naggs; ++a)
    if (plan.ops[a] != WS_AGG_COUNT && lay.kind[a] != SK_NONE) add(plan.aggs[a], out.aggs[a]);
  if (code.size() > sizeof(out.code) / sizeof(out.code[0])) throw Error("plan too large for the interpreter", WS_ERR_PLAN);
  memcpy(out.code, code.data(), code.size() * sizeof(TInstr));
}

EnvK envK(const ws_expr_env& env) {
  EnvK k;
  memcpy(k.consts, env.consts, sizeof k.consts);
  memcpy(k.sets, env.sets, sizeof k.sets);
  memcpy(k.setSize, env.setSize, sizeof k.setSize);
  memcpy(k.maps, env.maps, sizeof k.maps);
  memcpy(k.mapSize, env.mapSize, sizeof k.mapSize);
  k.ovf = env.ovf;
  return k;
}

}  // namespace ws
