// Launch-shape autotuner for the aggregation scans.  The choices are kept per key = (scan kernel,
// plan, size class): the plan is a 64-bit FNV-1a digest of the compiled evaluator's source (the
// interpreter: of the plan's shape), the size class log2 of the scan's tiles.  A choice is the CTAs
// per SM of the persistent grid (0: as many as fit), for the hash scan the shared-memory budget of the
// per-CTA table in KB (0: the default), and for compiled no-key and private-row scans the depth of the
// TMA tile staging (0: direct loads, 2..4 stages, -1: the default); for a hash join (keys `join:b<log2
// build keys>:p<log2 probe rows>`) the table's slots per build key (0: the default).  In tuning mode a
// key seen for the first time is tuned on the query's own data (aggRun in ws_ops.cu and joinImpl in
// ws_select_join.cu time each candidate and keep the fastest); the table lives in memory and, once a
// plan-cache directory is set, in <dir>/wsb200_tune.txt (one line per key: `key ctas smem_kb stages
// slots microseconds`; lines without the last fields are read with the defaults), read back when the
// directory is set.  No counterpart in the reference, whose launch shapes are fixed
// (src/gpu.cu:393-653).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "ws_b200.h"
#include "ws_internal.h"

namespace ws {
namespace {

struct Entry {
  TuneChoice c;
  double us = 0;
};

std::mutex gMu;
std::map<std::string, Entry> gTable;
std::string gFile;
int gMode = WS_TUNE_USE;

uint64_t fnv1a(const void* p, size_t n, uint64_t h = 0xcbf29ce484222325ull) {
  const unsigned char* b = (const unsigned char*)p;
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

bool parseLine(const std::string& line, std::string& key, Entry& e) {
  std::istringstream in(line);
  if (!(in >> key)) return false;
  std::vector<double> v;
  double x;
  while (in >> x) v.push_back(x);
  if (!in.eof() || v.size() < 3 || v.size() > 5) return false;
  const int ctas = (int)v[0], smem = (int)v[1], stages = v.size() >= 4 ? (int)v[2] : -1;
  const int slots = v.size() == 5 ? (int)v[3] : 0;
  if (v[0] != ctas || v[1] != smem || ctas < 0 || ctas > 64 || smem < 0 || smem > 228) return false;
  if (stages != -1 && stages != 0 && (stages < 2 || stages > 4)) return false;
  if (slots != 0 && (slots < 2 || slots > 16)) return false;
  e.c.ctasPerSm = ctas;
  e.c.smemKB = smem;
  e.c.stages = stages;
  e.c.slotsPerKey = slots;
  e.c.found = true;
  e.us = v.back();
  return true;
}

std::string formatLine(const std::string& key, const Entry& e) {
  char b[96];
  std::snprintf(b, sizeof(b), " %d %d %d %d %.1f\n", e.c.ctasPerSm, e.c.smemKB, e.c.stages, e.c.slotsPerKey, e.us);
  return key + b;
}

}  // namespace

int tuneMode() {
  std::lock_guard<std::mutex> l(gMu);
  return gMode;
}

std::string tuneKey(const char* kernel, const ws_jit_program* jit, const ws_agg_plan& plan, int64_t ntiles) {
  uint64_t h;
  if (jit) {
    h = fnv1a(jit->source.data(), jit->source.size());
  } else {
    const int shape[3] = {plan.nkeys, plan.naggs, plan.hasWhere};
    h = fnv1a(shape, sizeof(shape), 0x9e3779b97f4a7c15ull);
  }
  int cls = 0;
  while (cls < 62 && ((int64_t)1 << (cls + 1)) <= ntiles) ++cls;
  char b[96];
  std::snprintf(b, sizeof(b), "%s:%s%016llx:t%d", kernel, jit ? "q" : "i", (unsigned long long)h, cls);
  return b;
}

bool tuneLookup(const std::string& key, TuneChoice& c) {
  std::lock_guard<std::mutex> l(gMu);
  if (gMode == WS_TUNE_OFF) return false;
  auto it = gTable.find(key);
  if (it == gTable.end()) return false;
  c = it->second.c;
  return true;
}

void tuneStore(const std::string& key, const TuneChoice& c, double us) {
  std::lock_guard<std::mutex> l(gMu);
  Entry e;
  e.c = c;
  e.c.found = true;
  e.us = us;
  gTable[key] = e;
  if (!gFile.empty()) {
    std::ofstream f(gFile, std::ios::app);
    if (f) f << formatLine(key, e);
  }
}

void tuneSetDir(const std::string& dir) {
  std::lock_guard<std::mutex> l(gMu);
  gFile = dir.empty() ? std::string() : dir + "/wsb200_tune.txt";
  if (gFile.empty()) return;
  std::ifstream f(gFile);
  std::string line, key;
  while (std::getline(f, line)) {
    Entry e;
    if (parseLine(line, key, e)) gTable[key] = e;  // later lines win
  }
}

}  // namespace ws

extern "C" {

int ws_tune_set_mode(int mode) {
  if (mode != WS_TUNE_USE && mode != WS_TUNE_ON && mode != WS_TUNE_OFF) return WS_ERR_ARG;
  std::lock_guard<std::mutex> l(ws::gMu);
  ws::gMode = mode;
  return WS_OK;
}

int ws_tune_table(char* buf, size_t size, size_t* needed) {
  std::string s;
  {
    std::lock_guard<std::mutex> l(ws::gMu);
    for (const auto& kv : ws::gTable) s += ws::formatLine(kv.first, kv.second);
  }
  if (needed) *needed = s.size() + 1;
  if (buf && size) {
    const size_t n = std::min(size - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return buf && size < s.size() + 1 ? WS_ERR_SIZE : WS_OK;
}

int ws_tune_load(const char* text) {
  if (!text) return WS_ERR_ARG;
  std::istringstream in(text);
  std::string line, key;
  int bad = 0;
  std::lock_guard<std::mutex> l(ws::gMu);
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    ws::Entry e;
    if (ws::parseLine(line, key, e)) ws::gTable[key] = e;
    else ++bad;
  }
  return bad ? WS_ERR_ARG : WS_OK;
}

int ws_tune_clear(void) {
  std::lock_guard<std::mutex> l(ws::gMu);
  ws::gTable.clear();
  return WS_OK;
}

}  // extern "C"
