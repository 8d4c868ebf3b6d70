"""The drop-in check: the engine's own ABI headers (Warpstore src/devtypes.h, common.h through expr.h)
compiled together with include/ws_gpu.hpp in WS_GPU_ENGINE_TYPES mode, every field of the engine's
structs at the offset of its ws_* twin, and one translation unit that calls every src/gpu.h and
src/jit.h entry the engine's sources call, linked against libwarpstore_b200.so (the calls sit behind
a branch that never runs: no device is touched).  Skipped where the Warpstore sources are absent."""
import os
import subprocess

import pytest

from oracle import build_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = build_ref.REF_SRC

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REF_SRC, "devtypes.h")),
                                reason="the Warpstore sources are not on this machine")

FIELDS = {
    "Instr": ("ws_instr", ["op", "isInt", "arg"]),
    "ColView": ("ws_col_view", ["p", "t", "scale", "enc", "off"]),
    "Prog": ("ws_prog", ["start", "len"]),
    "ExprEnv": ("ws_expr_env", ["code", "consts", "sets", "setSize", "maps", "mapSize", "cols", "ovf"]),
    "AggPlan": ("ws_agg_plan", ["hasWhere", "where", "nkeys", "keys", "naggs", "aggs", "ops", "aggInt", "aggBits",
                                "aggPart", "aggNull", "densePriv", "keyInt", "genv"]),
    "DenseSpec": ("ws_dense_spec", ["G", "copies", "copyBytes", "priv", "kmin", "range", "stride", "slotOff", "kind"]),
}

CALLS = r"""
using namespace gdb;
static void everyEntry() {
  // device runtime (src/gpu.h:12-56)
  gpuInit(); (void)gpuSmCount(); (void)gpuArch(); (void)gpuDescribe();
  void* d = devAlloc(64); devFree(d);
  void* t = tmpAlloc(64); tmpFree(t); gpuTrimPool();
  char h[64] = {};
  h2d(d, h, 8); d2h(h, d, 8); d2d(d, d, 8); gpuSync();
  gpuSetVramLimit(1 << 30); (void)gpuVramUsed(); (void)gpuVramFill(); (void)gpuVramLimit(); (void)gpuVramFree();
  bool mapped = false;
  void* c = placeColumn(h, 64, mapped); releaseColumn(c, h, 64, mapped);
  c = placeColumn(h, 64, mapped, true); releaseColumn(c, h, 64, mapped);
  c = vramAcquire(h, 64); vramRelease(c, 64);
  c = hostMap(h, 64); hostUnmap(h);
  int32_t rows[1] = {0};
  int64_t vals[1] = {1};
  c = gpuPatchColumn(d, 64, 8, rows, vals, 1); vramRelease(c, 64);
  GpuUpdate u; u.kind = 2; u.add = 1; u.nul = kNullI64; u.lo = -10; u.hi = 10; u.notNull = true;
  c = gpuUpdateColumn(d, d, 8, 8, false, rows, 1, u); (void)u.bad; (void)u.sawNull; (void)u.mn; (void)u.mx;
  DevVec<int32_t> idx(16); std::vector<int32_t> back = idx.download(4);
  // aggregation (src/gpu.h:84-130)
  AggPlan plan{}; plan.naggs = 1; plan.ops[0] = AGG_COUNT;
  ExprEnv env{};
  DenseSpec ds{};
  GpuAggregator agg(plan, 1024, &ds);
  agg.addBatch(env, 1, 16, nullptr);
  agg.runWindow(env, nullptr);
  agg.run(env, nullptr);
  (void)agg.batches(); (void)agg.windows(); (void)agg.rowsIn(); (void)agg.dense(); (void)agg.capacity();
  if (agg.overflowed()) (void)agg.groupCount();
  std::vector<double> keys, accs;
  (void)agg.fetch(keys, accs);
  std::vector<uint8_t> sb = agg.sumBitsSlots(); const std::vector<int64_t>& hi = agg.sumHigh(); (void)hi;
  DevVec<double> dk, da; (void)agg.compact(dk, da);
  // selection, gathers, codes, evaluation (src/gpu.h:132-172)
  Prog where{0, 1};
  (void)gpuSelect(env, true, where, 16, nullptr, idx.p, nullptr);
  std::vector<int64_t> bn{16}, per;
  std::vector<const uint32_t*> bdel{nullptr};
  std::vector<ColView> bcols(1);
  DevVec<int32_t> sel;
  (void)gpuSelectMulti(env, true, where, bn, bdel, bcols, 1, sel, per, nullptr);
  gpuGatherMulti(bcols, bn, PType::I64, 8, idx.p, 4, d);
  gpuGather(d, PType::I32, idx.p, 4, d);
  gpuGatherEnc(bcols[0], PType::I64, idx.p, 4, d);
  gpuGatherNull(d, PType::F64, idx.p, 4, d);
  gpuGatherBytes(d, 16, idx.p, 4, d, true);
  gpuRemapCodes(idx.p, 4, idx.p, 4, idx.p);
  gpuBitsToDouble((const double*)d, 4, (double*)d);
  gpuEvalAt(env, where, idx.p, 4, (double*)d);
  gpuEvalAtInt(env, where, idx.p, 4, (int64_t*)d);
  std::vector<int64_t> distinct = gpuDistinctInts(env, where, idx.p, 4, 0, 100);
  bool sawNull = false;
  uint32_t* bits = gpuBitsFromColumn(d, 1, 4, 0, 64, &sawNull); devFree(bits);
  TempColSpec s; s.src = 1; s.kind = 4; s.cnt = 0; s.out = 2;
  double mn = 0, mx = 0;
  void* col = gpuTempColumn((const double*)d, 1, (const double*)d, 1, 4, s, mn, mx); devFree(col);
  gpuKeyBitmap(bcols[0], 4, 0, 64, (uint32_t*)d);
  gpuSetBits((uint32_t*)d, idx.p, 4);
  // joins (src/gpu.h:176-191)
  DevVec<int32_t> ob, op;
  (void)gpuHashJoin(bcols[0], 4, bcols[0], 4, ob, op);
  std::vector<int64_t> off;
  (void)gpuHashJoinParts(bcols[0], {0, 4}, bcols[0], {0, 4}, ob, op, &off);
  (void)gpuHashJoinOuter(bcols[0], 4, bcols[0], 4, ob, op, true);
  (void)gpuCrossJoin(2, 2, ob, op);
  // ORDER BY (src/gpu.h:197-201)
  DevVec<int32_t> perm = gpuSortPerm({{(const double*)d, false}}, 4);
  gpuMapRank((double*)d, idx.p, 4);
  std::vector<int32_t> hp = gpuSortPermHost(h, PType::I64, 4);
  // compiled plans (src/jit.h)
  (void)jitEnabled(); (void)jitMode(); jitSetMode(JIT_SYNC); jitSetDefaultMode(JIT_ON); jitSetCacheDir("");
  const JitProgram* jp = jitGet(env, 1, plan, JF_GROUPED, "aggregate");
  (void)jp; (void)JF_NOKEYS; (void)JF_DENSE; (void)JF_FLAG; (void)JF_FLAGM; (void)JIT_OFF;
  (void)progIsInt(env, where);
  jitBeginQuery("SELECT 1");
  JitQueryInfo ji = jitEndQuery(1.0);
  (void)ji.compiled; (void)ji.hits; (void)ji.fromDisk; (void)ji.background; (void)ji.compileMs; (void)ji.ids.size();
  for (auto& r : jitPlanCache())
    (void)(r.id + r.kind.size() + r.origin.size() + r.compileMs + r.execs + r.avgMs + r.lastMs + r.sourceBytes + r.sql.size());
  std::string src = jitSourceOf(1);
  jitClearCache();
}
int main(int argc, char**) {
  if (argc > 99) everyEntry();  // linked, never run: no device is touched
  return 0;
}
"""


def test_engine_headers_and_every_entry_link(built, tmp_path):
    lines = ['#include "expr.h"  // the engine\'s common.h + devtypes.h', "#include <cstddef>",
             "#define WS_GPU_ENGINE_TYPES 1", '#define WS_GPU_THROW(m, c) throw gdb::SqlError((m), (c))',
             '#include "ws_gpu.hpp"']
    for eng, (ws, fields) in FIELDS.items():
        lines.append(f"static_assert(sizeof(gdb::{eng}) == sizeof({ws}), \"sizeof {eng}\");")
        for f in fields:
            lines.append(f"static_assert(offsetof(gdb::{eng}, {f}) == offsetof({ws}, {f}), \"{eng}::{f}\");")
    src = tmp_path / "engine_link.cpp"
    src.write_text("\n".join(lines) + "\n" + CALLS)
    exe = tmp_path / "engine_link"
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wno-unused-variable", "-I", REF_SRC, "-I",
                        os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L",
                        os.path.join(ROOT, "warpstore_b200"), "-lwarpstore_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "warpstore_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    assert subprocess.run([str(exe)]).returncode == 0
