"""The C-ABI library loads on a host without a GPU, exports every function include/*.h declares, and
agrees with the Python mirror on the layout of the engine's structs."""
import ctypes as C
import os
import re

import pytest

from warpstore_b200 import abi
from warpstore_b200._lib import LIB_PATH, SIGNATURES, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("ws_b200.h",):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(ws_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_loads(built):
    assert os.path.exists(LIB_PATH)
    lib()


def test_exports_every_declared_symbol(built):
    l = C.CDLL(LIB_PATH)
    declared = declared_functions()
    assert len(declared) > 40
    missing = [n for n in declared if not hasattr(l, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert declared <= set(SIGNATURES), f"no Python signature for: {declared - set(SIGNATURES)}"


def test_struct_layout_matches(built):
    n = 64
    out = (C.c_int64 * n)()
    m = lib().ws_abi_layout(out, n)
    assert list(out)[:m] == abi.layout()
    # the engine's layout (src/devtypes.h): sizes pinned
    assert C.sizeof(abi.ExprEnv) == 4488 and C.sizeof(abi.AggPlan) == 648 and C.sizeof(abi.DenseSpec) == 536


def test_no_device_is_reported_not_crashed(built):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    rc = lib().ws_gpu_init()
    assert rc != 0
    assert lib().ws_last_error()


def test_jit_modes_are_per_thread(built):
    import threading
    l = lib()
    l.ws_jit_set_mode(abi.JIT_SYNC)
    seen = []
    t = threading.Thread(target=lambda: seen.append(l.ws_jit_mode()))
    t.start()
    t.join()
    assert l.ws_jit_mode() == abi.JIT_SYNC
    assert seen[0] == abi.JIT_ON  # the default
    l.ws_jit_set_mode(-1)


def test_cpp_shim_compiles_and_links(built, tmp_path):
    """include/ws_gpu.hpp (the engine-side C++ interface over the C ABI) compiles and links."""
    import subprocess
    src = tmp_path / "shim.cpp"
    src.write_text('''
#include "ws_gpu.hpp"
#include <cstdio>
int main() {
  gdb::AggPlan plan{};
  plan.naggs = 1;
  plan.ops[0] = WS_AGG_COUNT;
  try {
    gdb::gpuInit();
    gdb::GpuAggregator agg(plan, 1024);
    std::vector<double> k, a;
    agg.fetch(k, a);
  } catch (const gdb::WsGpuError& e) {
    std::printf("error %d\\n", e.code);
  }
  return 0;
}
''')
    exe = tmp_path / "shim"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", os.path.join(ROOT, "warpstore_b200"), "-lwarpstore_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "warpstore_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
