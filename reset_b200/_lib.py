"""ctypes binding of libreset.so (the C ABI declared in include/reset.h).

The library is loaded from this package directory.  There is no fallback:
if libreset.so is missing or cannot be loaded, importing the bindings
raises, so no code path silently runs without the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libreset.so")

STATUS = {
    0: "RESET_OK", 1: "RESET_ERR_CUDA", 2: "RESET_ERR_OOM", 3: "RESET_ERR_ARG",
    4: "RESET_ERR_TABLE_FULL", 5: "RESET_ERR_PROBE_LIMIT",
    6: "RESET_ERR_TIMEOUT", 7: "RESET_ERR_UNSUPPORTED", 8: "RESET_ERR_BUSY",
}


class ResetError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("alpha", C.c_float), ("bucket", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class Tuning(C.Structure):
    _fields_ = [("probe_rounds", C.c_int32), ("warp_pair_min", C.c_int32),
                ("probe_variant", C.c_int32), ("pair_method", C.c_int32),
                ("reserved", C.c_int32 * 4)]


class TableView(C.Structure):
    _fields_ = [("n", C.c_int32), ("bucket", C.c_int32), ("max_len", C.c_int32),
                ("hierarchical", C.c_int32), ("bucket_num", C.c_int64),
                ("m", C.c_int64), ("alpha", C.c_float), ("pad", C.c_int32),
                ("d_table", C.c_void_p), ("d_len", C.c_void_p),
                ("d_off", C.c_void_p)]


class Pattern(C.Structure):
    _fields_ = [("k", C.c_int32), ("flags", C.c_int32),
                ("offsets", C.POINTER(C.c_int32)), ("backward", C.POINTER(C.c_int32)),
                ("restriction", C.POINTER(C.c_int32)), ("reuse", C.POINTER(C.c_int32))]


class ServerConfig(C.Structure):
    _fields_ = [("streams", C.c_int32), ("max_batch_requests", C.c_int32),
                ("mem_budget_bytes", C.c_int64), ("max_batch_cost", C.c_int64),
                ("pinned_result_bytes", C.c_int64), ("reserved", C.c_int32 * 4)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int32), ("index", C.c_int32),
                ("args", C.POINTER(C.c_int32)), ("nargs", C.c_int64),
                ("args2", C.POINTER(C.c_int32)), ("nargs2", C.c_int64),
                ("num", C.c_int32), ("den", C.c_int32), ("arrival_ns", C.c_int64),
                ("reserved", C.c_int32 * 4)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("kind", C.c_int32), ("count", C.c_int64),
                ("docs", C.POINTER(C.c_int32)), ("ndocs", C.c_int64),
                ("values", C.POINTER(C.c_int64)), ("nvalues", C.c_int64),
                ("flags", C.POINTER(C.c_uint8)), ("queue_us", C.c_double),
                ("service_us", C.c_double), ("latency_us", C.c_double),
                ("batch_id", C.c_int64), ("batch_size", C.c_int32),
                ("reserved", C.c_int32)]


class ServerCounters(C.Structure):
    _fields_ = [("completed", C.c_int64), ("batches", C.c_int64),
                ("max_batch", C.c_int64), ("pending", C.c_int64),
                ("inflight_batches", C.c_int64), ("max_inflight_batches", C.c_int64),
                ("budget_bytes", C.c_int64), ("in_use_bytes", C.c_int64),
                ("max_in_use_bytes", C.c_int64), ("mean_batch", C.c_double),
                ("launch_host_us", C.c_double), ("batch_us", C.c_double),
                ("arena_bytes", C.c_int64), ("max_launch_us", C.c_double),
                ("max_finish_us", C.c_double), ("reserved", C.c_int64 * 2)]


P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64

# name -> (restype, argtypes); every symbol include/reset.h declares.
SIGNATURES = {
    "reset_params_default": (None, [C.POINTER(Params)]),
    "reset_table_build": (I32, [P, P, I32, I64, C.POINTER(Params), I32, P,
                                C.POINTER(P), P]),
    "reset_table_info": (I32, [P, C.POINTER(TableView)]),
    "reset_table_free": (I32, [P]),
    "reset_table_free_async": (I32, [P, P]),
    "reset_release_cached_memory": (I32, []),
    "reset_table_check": (I32, [P, P]),
    "reset_csr_hash_order": (I32, [P, P, P, P]),
    "reset_tc_count": (I32, [P, P, P, I64, P, P]),
    "reset_tc_count_ex": (I32, [P, P, P, I64, I32, P, P]),
    "reset_tc_count_noalloc": (I32, [P, P, P, I64, P, P]),
    "reset_tc_count_batch": (I32, [P, P, P, I64, P, I32, P, P]),
    "reset_clique4_count": (I32, [P, P, P, I64, P, P]),
    "reset_clique_count": (I32, [P, P, P, I64, I32, P, P]),
    "reset_pattern_count": (I32, [P, P, P, I64, C.POINTER(Pattern), P, P]),
    "reset_pattern_named": (I32, [C.c_char_p, C.POINTER(Pattern), C.POINTER(C.c_int32)]),
    "reset_sss": (I32, [P, P, P, P, P, I64, I32, I32, P, P, P]),
    "reset_sss_float": (I32, [P, P, P, P, P, I64, C.c_float, P, P, P]),
    "reset_ir": (I32, [P, P, P, P, P, I32, P, P, P, P]),
    "reset_intersect_count": (I32, [P, I64, P, I64, C.POINTER(Params), P, P]),
    "reset_csr_shard": (I32, [P, P, I32, I64, I32, I32, P, P, P, P]),
    "reset_tc_count_shard": (I32, [P, P, P, I64, P, P, I64, P, P]),
    "reset_sss_decide": (I32, [P, I32, P, P, I64, P, I32, I32, P, P, P]),
    "reset_gen_rmat": (I32, [I32, I32, C.c_uint64, C.c_double, C.c_double,
                             C.c_double, I32, C.POINTER(P), C.POINTER(P),
                             C.POINTER(I64), P]),
    "reset_batch_create": (I32, [P, P, I64, I32, I32, C.POINTER(P), P]),
    "reset_batch_create_ex": (I32, [P, P, I64, I32, I32, I32, C.POINTER(P), P]),
    "reset_batch_buffers": (I32, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                  C.POINTER(P)]),
    "reset_batch_run": (I32, [P, I64, P]),
    "reset_batch_destroy": (I32, [P]),
    "reset_gen_token_sets": (I32, [I32, I32, C.c_double, I32, I32, C.c_double,
                                   C.c_double, C.c_uint64,
                                   C.POINTER(P), C.POINTER(P), C.POINTER(I64), P]),
    "reset_prefix_candidates": (I32, [P, P, I32, I64, I32, I32, I32, C.POINTER(P),
                                      C.POINTER(P), C.POINTER(I64), P]),
    "reset_gen_inverted_index": (I32, [I32, I32, C.c_double, I64, C.c_uint64,
                                       C.POINTER(P), C.POINTER(P), C.POINTER(I64), P]),
    "reset_server_config_default": (None, [C.POINTER(ServerConfig)]),
    "reset_now_ns": (I64, []),
    "reset_server_create": (I32, [C.POINTER(ServerConfig), C.POINTER(P)]),
    "reset_server_add_index": (I32, [P, P, P, P, C.POINTER(I32)]),
    "reset_server_submit": (I32, [P, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "reset_server_wait": (I32, [P, C.c_uint64, I32, C.POINTER(Result)]),
    "reset_server_release": (I32, [P, C.c_uint64]),
    "reset_server_stats": (I32, [P, C.POINTER(ServerCounters)]),
    "reset_server_destroy": (I32, [P]),
    "reset_free": (I32, [P]),
    "reset_last_error_string": (C.c_char_p, []),
    "reset_status_string": (C.c_char_p, [I32]),
    "reset_abi_version": (I32, []),
    "reset_get_tuning": (I32, [C.POINTER(Tuning)]),
    "reset_set_tuning": (I32, [C.POINTER(Tuning)]),
    "reset_kernel_launches": (I64, []),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libreset.so and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"libreset.so not found at {path}; build it with "
            "`python -m reset_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != 0:
        msg = load().reset_last_error_string()
        raise ResetError(status, msg.decode() if msg else "")
