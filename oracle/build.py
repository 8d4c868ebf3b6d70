"""Builds the CPU oracle (test infrastructure): oracle/libws_oracle.so from oracle/ws_oracle.cpp with g++."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libws_oracle.so")
SRC = os.path.join(HERE, "ws_oracle.cpp")
HDRS = [os.path.join(HERE, "ws_oracle.h"), os.path.join(os.path.dirname(HERE), "include", "ws_types.h")]


def build() -> str:
    deps = [SRC] + HDRS
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-Wall", SRC, "-o", LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build())
