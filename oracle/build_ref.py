"""Recipe: the reference's own GPU operators — Warpstore src/gpu.cu and src/jit.cu with the headers they
include, read where they lie under /root/reference — + oracle/ref_harness.cu -> oracle/_ref/libwsref.so,
for sm_100a.  Test infrastructure only.  Builds nothing when the reference sources are not on this
machine (the GPU box uses the library built here).

src/jit.cu includes a header that the reference's CMake build generates (cmake/embed.cmake): its
devtypes.h and kernels.cuh as two C++ raw string literals, the sources its run-time compiler feeds to
NVRTC.  This recipe writes that header itself (oracle/_ref/gen/jit_sources.h, the same two literals)
rather than running the reference's build system.  The library links NVRTC and the driver API, as the
reference's executable does."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")
LIB = os.path.join(OUT, "libwsref.so")
# the Warpstore source tree's src/ directory (read where it lies; WARPSTORE_REFERENCE_SRC overrides)
REF_SRC = os.environ.get("WARPSTORE_REFERENCE_SRC", "/root/reference/src")


def _embed_header() -> str:
    """oracle/_ref/gen/jit_sources.h: gdb::kJitDevtypesSrc / kJitKernelsSrc as raw string literals."""
    a = open(os.path.join(REF_SRC, "devtypes.h")).read()
    b = open(os.path.join(REF_SRC, "kernels.cuh")).read()
    for t in (a, b):
        if ')GDBSRC"' in t:
            raise RuntimeError("the reference sources contain the literal's delimiter")
    text = ("// Written by oracle/build_ref.py: the reference's device sources for its run-time compiler.\n"
            "#pragma once\nnamespace gdb {\n"
            f'static const char* const kJitDevtypesSrc = R"GDBSRC({a})GDBSRC";\n'
            f'static const char* const kJitKernelsSrc = R"GDBSRC({b})GDBSRC";\n'
            "}  // namespace gdb\n")
    os.makedirs(GEN, exist_ok=True)
    path = os.path.join(GEN, "jit_sources.h")
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)
    return path


def build() -> str | None:
    if not os.path.exists(os.path.join(REF_SRC, "gpu.cu")):
        return LIB if os.path.exists(LIB) else None
    harness = os.path.join(HERE, "ref_harness.cu")
    deps = [os.path.join(REF_SRC, f) for f in ("gpu.cu", "jit.cu", "gpu.h", "jit.h", "kernels.cuh", "devtypes.h",
                                               "common.h", "expr.h")] + [harness, os.path.abspath(__file__)]
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    os.makedirs(OUT, exist_ok=True)
    _embed_header()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    flags = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "--default-stream", "per-thread",
             "--expt-relaxed-constexpr", "-DCUDA_API_PER_THREAD_DEFAULT_STREAM=1", "-Xcompiler", "-fPIC",
             "-I", REF_SRC, "-I", GEN]
    objs = []
    for src, obj in ((os.path.join(REF_SRC, "gpu.cu"), "gpu.o"), (os.path.join(REF_SRC, "jit.cu"), "jit.o"),
                     (harness, "ref_harness.o")):
        o = os.path.join(OUT, obj)
        r = subprocess.run([nvcc, "-c", src, "-o", o] + flags, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed for {src}:\n{r.stderr}")
        objs.append(o)
    # libcuda: the driver's stub library links here (no driver in this container); the box has the driver
    stubs = os.path.join(cuda, "lib64", "stubs")
    r = subprocess.run([nvcc, "-shared", "-o", LIB] + objs +
                       ["-gencode", "arch=compute_100a,code=sm_100a", "-L", os.path.join(cuda, "lib64"), "-L", stubs,
                        "-lcudart", "-lnvrtc", "-lcuda", "-Xlinker", "-rpath," + os.path.join(cuda, "lib64")],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference link failed:\n{r.stderr}")
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build())
