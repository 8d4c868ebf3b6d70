"""Recipe: the reference's own GPU operators (Warpstore src/gpu.cu and the headers it includes, read
where they lie under /root/reference) + oracle/ref_harness.cu -> oracle/_ref/libwsref.so, for sm_100a.
Test infrastructure only.  Builds nothing when the reference sources are not on this machine (the GPU
box uses the library built here)."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libwsref.so")
REF_SRC = "/root/reference/src"


def build() -> str | None:
    if not os.path.exists(os.path.join(REF_SRC, "gpu.cu")):
        return LIB if os.path.exists(LIB) else None
    harness = os.path.join(HERE, "ref_harness.cu")
    deps = [os.path.join(REF_SRC, f) for f in ("gpu.cu", "gpu.h", "jit.h", "kernels.cuh", "devtypes.h", "common.h",
                                               "expr.h")] + [harness]
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    os.makedirs(OUT, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    flags = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "--default-stream", "per-thread",
             "--expt-relaxed-constexpr", "-DCUDA_API_PER_THREAD_DEFAULT_STREAM=1", "-Xcompiler", "-fPIC",
             "-I", REF_SRC]
    objs = []
    for src, obj in ((os.path.join(REF_SRC, "gpu.cu"), "gpu.o"), (harness, "ref_harness.o")):
        o = os.path.join(OUT, obj)
        r = subprocess.run([nvcc, "-c", src, "-o", o] + flags, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed for {src}:\n{r.stderr}")
        objs.append(o)
    r = subprocess.run([nvcc, "-shared", "-o", LIB] + objs + ["-gencode", "arch=compute_100a,code=sm_100a", "-lcudart"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference link failed:\n{r.stderr}")
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build())
