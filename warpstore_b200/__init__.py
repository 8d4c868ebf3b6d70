"""warpstore_b200 — B200-native query-execution core for the Warpstore engine's analytic hot path.

The product is libwarpstore_b200.so (C ABI in include/ws_b200.h, built by warpstore_b200/build.py):
fused scan / filter / aggregate over column segments, dense and hash GROUP BY, selection, gathers and
hash joins as sm_100a kernels generated per query with NVRTC.  This package is the thin Python mirror
of the engine's operator interface used by the tests and the benchmark.
"""
from . import abi, query  # noqa: F401
from ._lib import LIB_PATH, WsError, lib  # noqa: F401
from .ops import *  # noqa: F401,F403
