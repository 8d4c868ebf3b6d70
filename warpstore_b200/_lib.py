"""Loads libwarpstore_b200.so (built in-tree) and declares the C ABI of include/ws_b200.h.

The product path has no fallback: if the shared library is missing or cannot be loaded, every
operator raises.  Build it with `python warpstore_b200/build.py` (or __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwarpstore_b200.so")

P = C.c_void_p
I64P = C.POINTER(C.c_int64)

# name: (restype, argtypes)
SIGNATURES = {
    "ws_last_error": (C.c_char_p, []),
    "ws_last_error_code": (C.c_int, []),
    "ws_gpu_init": (C.c_int, []),
    "ws_gpu_sm_count": (C.c_int, []),
    "ws_gpu_arch": (C.c_int, []),
    "ws_gpu_describe": (C.c_int, [C.c_char_p, C.c_size_t]),
    "ws_set_stream": (C.c_int, [P]),
    "ws_get_stream": (P, []),
    "ws_dev_alloc": (C.c_int, [C.c_size_t, C.POINTER(P)]),
    "ws_dev_free": (C.c_int, [P]),
    "ws_tmp_alloc": (C.c_int, [C.c_size_t, C.POINTER(P)]),
    "ws_tmp_free": (C.c_int, [P]),
    "ws_h2d": (C.c_int, [P, P, C.c_size_t]),
    "ws_d2h": (C.c_int, [P, P, C.c_size_t]),
    "ws_d2d": (C.c_int, [P, P, C.c_size_t]),
    "ws_gpu_sync": (C.c_int, []),
    "ws_gpu_trim_pool": (C.c_int, []),
    "ws_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(P)]),
    "ws_host_free": (C.c_int, [P]),
    "ws_set_vram_limit": (C.c_int, [C.c_int64]),
    "ws_vram_used": (C.c_int64, []),
    "ws_vram_limit": (C.c_int64, []),
    "ws_vram_free": (C.c_int64, []),
    "ws_vram_fill": (C.c_double, []),
    "ws_place_column": (C.c_int, [P, C.c_size_t, C.c_int, C.POINTER(P), C.POINTER(C.c_int)]),
    "ws_release_column": (C.c_int, [P, P, C.c_size_t, C.c_int]),
    "ws_vram_acquire": (C.c_int, [P, C.c_size_t, C.POINTER(P)]),
    "ws_vram_release": (C.c_int, [P, C.c_size_t]),
    "ws_host_map": (C.c_int, [P, C.c_size_t, C.POINTER(P)]),
    "ws_host_unmap": (C.c_int, [P]),
    "ws_patch_column": (C.c_int, [P, C.c_size_t, C.c_int, P, P, C.c_int64, C.POINTER(P)]),
    "ws_update_column": (C.c_int, [P, P, C.c_int64, C.c_int, C.c_int, P, C.c_int64, C.POINTER(abi.Update),
                                   C.POINTER(P)]),
    "ws_distinct_ints": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, P, C.c_int64, C.c_int64, C.c_int64, P,
                                   C.c_int64, I64P]),
    "ws_bits_from_column": (C.c_int, [P, C.c_int, C.c_int64, C.c_int64, C.c_int64, C.POINTER(P), C.POINTER(C.c_int)]),
    "ws_temp_column": (C.c_int, [P, C.c_int, P, C.c_int, C.c_int64, C.POINTER(abi.TempColSpec), C.POINTER(P),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ws_sort_perm_host": (C.c_int, [P, C.c_int, C.c_int64, P]),
    "ws_jit_plan_text": (C.c_int, [C.c_int, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ws_jit_last_query_plans": (C.c_int, [P, C.c_int, C.POINTER(C.c_int)]),
    "ws_encode_column_engine": (C.c_int, [P, C.c_int, C.c_int64, C.POINTER(P), I64P, C.POINTER(C.c_int)]),
    "ws_agg_create": (C.c_int, [C.POINTER(abi.AggPlan), C.c_int64, C.POINTER(abi.DenseSpec), C.POINTER(P)]),
    "ws_agg_destroy": (None, [P]),
    "ws_agg_add_batch": (C.c_int, [P, C.POINTER(abi.ExprEnv), C.c_int, C.c_int64, P]),
    "ws_agg_add_batches": (C.c_int, [P, C.c_int, C.c_int, P, P, P]),
    "ws_agg_run": (C.c_int, [P, C.POINTER(abi.ExprEnv), P]),
    "ws_agg_run_many": (C.c_int, [P, P, P, C.c_int]),
    "ws_agg_run_window": (C.c_int, [P, C.POINTER(abi.ExprEnv), P]),
    "ws_agg_batches": (C.c_int, [P]),
    "ws_agg_windows": (C.c_int, [P]),
    "ws_agg_rows_in": (C.c_int64, [P]),
    "ws_agg_is_dense": (C.c_int, [P]),
    "ws_agg_capacity": (C.c_int64, [P]),
    "ws_agg_overflowed": (C.c_int, [P, C.POINTER(C.c_int)]),
    "ws_agg_group_count": (C.c_int, [P, I64P]),
    "ws_agg_fetch": (C.c_int, [P, C.c_int64, P, P, P, I64P]),
    "ws_agg_fetch_async": (C.c_int, [P, C.c_int64, C.c_int64, P, P, P]),
    "ws_exec_create": (C.c_int, [P, C.c_int64, P, P, C.c_int, C.c_int, P, P, P, P, C.c_int64, C.POINTER(P)]),
    "ws_exec_run": (C.c_int, [P, P]),
    "ws_exec_results": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "ws_exec_destroy": (None, [P]),
    "ws_exec_group_create": (C.c_int, [P, C.c_int, P, C.POINTER(P)]),
    "ws_exec_group_run": (C.c_int, [P, P]),
    "ws_exec_group_destroy": (None, [P]),
    "ws_agg_sum_bits_slots": (C.c_int, [P, P]),
    "ws_agg_sum_high": (C.c_int, [P, P]),
    "ws_agg_compact": (C.c_int, [P, C.POINTER(P), C.POINTER(P), I64P]),
    "ws_agg_nokeys_noalloc": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), P, C.c_int, P, P,
                                        P, P]),
    "ws_select": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, C.c_int64, P, P, P, I64P]),
    "ws_select_multi": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, C.c_int, P, P, P, C.c_int,
                                  C.POINTER(P), P, P, I64P]),
    "ws_gather_multi": (C.c_int, [P, P, C.c_int, C.c_int, C.c_int, P, C.c_int64, P]),
    "ws_gather": (C.c_int, [P, C.c_int, P, C.c_int64, P]),
    "ws_hash_join_parts": (C.c_int, [abi.ColView, P, C.c_int, abi.ColView, P, C.c_int, C.POINTER(P), C.POINTER(P),
                                     P, I64P]),
    "ws_hash_join": (C.c_int, [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.POINTER(P), C.POINTER(P), I64P]),
    "ws_hash_join_sized": (C.c_int, [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.c_int64, C.POINTER(P),
                                     C.POINTER(P), I64P, C.POINTER(C.c_int)]),
    "ws_hash_join_outer": (C.c_int, [abi.ColView, C.c_int64, abi.ColView, C.c_int64, C.c_int, C.POINTER(P),
                                     C.POINTER(P), I64P]),
    "ws_cross_join": (C.c_int, [C.c_int64, C.c_int64, C.POINTER(P), C.POINTER(P), I64P]),
    "ws_key_bitmap": (C.c_int, [abi.ColView, C.c_int64, C.c_int64, C.c_int64, P]),
    "ws_set_bits": (C.c_int, [P, P, C.c_int64]),
    "ws_remap_codes": (C.c_int, [P, C.c_int64, P, C.c_int64, P]),
    "ws_bits_to_double": (C.c_int, [P, C.c_int64, P]),
    "ws_gather_null": (C.c_int, [P, C.c_int, P, C.c_int64, P]),
    "ws_gather_bytes": (C.c_int, [P, C.c_int, P, C.c_int64, P, C.c_int]),
    "ws_gather_enc": (C.c_int, [abi.ColView, C.c_int, P, C.c_int64, P]),
    "ws_eval_at": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, P, C.c_int64, P]),
    "ws_eval_at_int": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, abi.Prog, P, C.c_int64, P]),
    "ws_sort_perm": (C.c_int, [P, P, C.c_int, C.c_int64, C.POINTER(P)]),
    "ws_map_rank": (C.c_int, [P, P, C.c_int64]),
    "ws_encode_column": (C.c_int, [P, C.c_int, C.c_int64, C.c_int, C.POINTER(P), I64P, C.POINTER(C.c_int)]),
    "ws_hll_sketch": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), C.c_int, P, P, P, C.c_int,
                                C.c_int64, P, I64P, I64P]),
    "ws_join_key_sample": (C.c_int, [abi.ColView, C.c_int64, C.c_uint64, P, C.c_int64, I64P]),
    "ws_mlp_infer": (C.c_int, [P, C.c_int, C.c_int, C.c_int, P, P, P, P, P, C.c_float, P]),
    "ws_serve": (C.c_int, [P, C.c_int, P, C.POINTER(C.c_double)]),
    "ws_tune_set_mode": (C.c_int, [C.c_int]),
    "ws_tune_table": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ws_tune_load": (C.c_int, [C.c_char_p]),
    "ws_tune_clear": (C.c_int, []),
    "ws_jit_set_mode": (C.c_int, [C.c_int]),
    "ws_jit_mode": (C.c_int, []),
    "ws_jit_set_default_mode": (C.c_int, [C.c_int]),
    "ws_jit_set_cache_dir": (C.c_int, [C.c_char_p]),
    "ws_jit_get": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), C.c_int, C.c_char_p,
                             C.POINTER(P)]),
    "ws_prog_is_int": (C.c_int, [C.POINTER(abi.ExprEnv), abi.Prog]),
    "ws_jit_program_info": (C.c_int, [P, C.POINTER(abi.JitInfo)]),
    "ws_jit_source_of": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ws_jit_plan_cache_count": (C.c_int, []),
    "ws_jit_plan_cache_row": (C.c_int, [C.c_int, C.POINTER(abi.JitInfo)]),
    "ws_jit_clear_cache": (C.c_int, []),
    "ws_jit_begin_query": (C.c_int, [C.c_char_p]),
    "ws_jit_end_query": (C.c_int, [C.c_double, C.POINTER(abi.JitQueryInfo)]),
    "ws_codegen_source": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), C.c_int, C.c_char_p,
                                    C.c_size_t, C.POINTER(C.c_size_t)]),
    "ws_codegen_compile_check": (C.c_int, [C.POINTER(abi.ExprEnv), C.c_int, C.POINTER(abi.AggPlan), C.c_int, C.c_int,
                                           C.POINTER(C.c_size_t)]),
    "ws_abi_layout": (C.c_int, [I64P, C.c_int]),
    "ws_kernel_launches": (C.c_int64, []),
}

_lib = None


class WsError(RuntimeError):
    """An operator failed; .code is the engine's SQL error number (1041 out of memory, 1105 internal ...)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run warpstore_b200/build.py")
        lb = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lb, name)
            f.restype = res
            f.argtypes = args
        _lib = lb
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        l = lib()
        raise WsError(rc, (l.ws_last_error() or b"").decode(errors="replace"))
