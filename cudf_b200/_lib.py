"""ctypes binding of the engine's C ABI (include/cudf_b200.h).

The shared library is built in-tree (cudf_b200/_build/libcudf_b200.so) by
``python -m cudf_b200.build``.  There is no CPU fallback: if the library is
missing or cannot load, every call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CUDF_B200_LIB", os.path.join(HERE, "_build", "libcudf_b200.so"))

GB_OK, GB_ERR_LOGIC, GB_ERR_CUDA, GB_ERR_ALLOC, GB_ERR_UNSUPPORTED = 0, 1, 2, 3, 4


class GbColumn(ctypes.Structure):
    _fields_ = [("type_id", ctypes.c_int32), ("size", ctypes.c_int64), ("data", ctypes.c_void_p),
                ("null_mask", ctypes.c_void_p), ("offset", ctypes.c_int64)]


class GbAgg(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("param", ctypes.c_int32)]


class GbRequest(ctypes.Structure):
    _fields_ = [("values", GbColumn), ("num_aggs", ctypes.c_int32), ("aggs", ctypes.POINTER(GbAgg))]


class GbOutColumn(ctypes.Structure):
    _fields_ = [("type_id", ctypes.c_int32), ("size", ctypes.c_int64), ("data", ctypes.c_void_p),
                ("null_mask", ctypes.c_void_p), ("null_count", ctypes.c_int64)]


class GbResult(ctypes.Structure):
    _fields_ = [("num_groups", ctypes.c_int64), ("num_keys", ctypes.c_int32),
                ("keys", ctypes.POINTER(GbOutColumn)), ("num_requests", ctypes.c_int32),
                ("num_results", ctypes.POINTER(ctypes.c_int32)),
                ("results", ctypes.POINTER(ctypes.POINTER(GbOutColumn))), ("impl", ctypes.c_void_p)]


class GbTuning(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("smem_bytes", ctypes.c_int32), ("smem_fill_pct", ctypes.c_int32),
                ("smem_max_groups", ctypes.c_int64), ("load_factor_pct", ctypes.c_int32),
                ("force_mode", ctypes.c_int32), ("groups_hint", ctypes.c_int64),
                ("profile", ctypes.c_int32), ("scatter", ctypes.c_int32), ("pass2", ctypes.c_int32),
                ("part_fill_pct", ctypes.c_int32), ("wagg_pct", ctypes.c_int32)]


class GbStats(ctypes.Structure):
    _fields_ = [("est_groups", ctypes.c_int64), ("capacity", ctypes.c_int64), ("mode", ctypes.c_int32),
                ("retries", ctypes.c_int32), ("kernels", ctypes.c_int32),
                ("agg_kernel_ms", ctypes.c_double), ("compact_ms", ctypes.c_double),
                ("scatter_ms", ctypes.c_double), ("rule", ctypes.c_int32)]


class GbTuningRule(ctypes.Structure):
    _fields_ = [("max_rows", ctypes.c_int64), ("max_groups", ctypes.c_int64), ("key_words", ctypes.c_int32),
                ("tuning", GbTuning)]


class GbBatchStats(ctypes.Structure):
    _fields_ = [("instances", ctypes.c_int64), ("tiles", ctypes.c_int64), ("smem_instances", ctypes.c_int64),
                ("table_bytes", ctypes.c_int64), ("output_bytes", ctypes.c_int64),
                ("kernels_per_run", ctypes.c_int32), ("regrown", ctypes.c_int64), ("block", ctypes.c_int32),
                ("tile_rows", ctypes.c_int64), ("ruled_instances", ctypes.c_int64)]


class GbBatchRule(ctypes.Structure):
    _fields_ = [("max_rows", ctypes.c_int64), ("max_groups", ctypes.c_int64), ("smem_slots", ctypes.c_int32),
                ("headroom_pct", ctypes.c_int32)]


class GbBatchLaunch(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("tile_rows", ctypes.c_int32), ("smem_bytes", ctypes.c_int32)]


class GbServerOptions(ctypes.Structure):
    _fields_ = [("memory_cap_bytes", ctypes.c_int64), ("max_batch_queries", ctypes.c_int32),
                ("max_batch_rows", ctypes.c_int64), ("workers", ctypes.c_int32),
                ("direct_rows", ctypes.c_int64), ("direct_groups", ctypes.c_int64),
                ("reserve_bytes", ctypes.c_int64)]


class GbQueryInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("latency_s", ctypes.c_double), ("queue_s", ctypes.c_double),
                ("num_groups", ctypes.c_int64)]


class GbServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double), ("queries_per_s", ctypes.c_double),
                ("peak_admitted_bytes", ctypes.c_int64), ("sketch_s", ctypes.c_double),
                ("prepare_s", ctypes.c_double), ("run_s", ctypes.c_double), ("trial_rounds", ctypes.c_int64),
                ("direct_runs", ctypes.c_int64), ("held_for_memory", ctypes.c_int64),
                ("min_free_bytes", ctypes.c_int64)]


class GroupbyError(RuntimeError):
    """A failure reported by the engine; ``code`` is the GB_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class LogicError(GroupbyError, ValueError):
    """cudf::logic_error (invalid arguments, size mismatch, invalid type/aggregation)."""


class CudaError(GroupbyError):
    """cudf::cuda_error."""


_lib = None

# declared C ABI: name -> (restype, argtypes)
SIGNATURES = {
    "gb_create": (ctypes.c_int, [ctypes.POINTER(GbColumn), ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "gb_aggregate": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbRequest), ctypes.c_int32,
                                    ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.POINTER(GbResult))]),
    "gb_result_free": (None, [ctypes.POINTER(GbResult)]),
    "gb_destroy": (None, [ctypes.c_void_p]),
    "gb_last_error": (ctypes.c_char_p, []),
    "gb_target_type": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32]),
    "gb_is_valid_aggregation": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32]),
    "gb_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbTuning)]),
    "gb_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbStats)]),
    "gb_set_tuning_rules": (ctypes.c_int, [ctypes.POINTER(GbTuningRule), ctypes.c_int32]),
    "gb_version": (ctypes.c_char_p, []),
    "gb_batch_prepare": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(GbColumn), ctypes.c_int32, ctypes.c_int32,
                                        ctypes.POINTER(GbRequest), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "gb_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "gb_batch_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(GbOutColumn), ctypes.POINTER(GbOutColumn)]),
    "gb_batch_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbBatchStats)]),
    "gb_batch_destroy": (None, [ctypes.c_void_p]),
    "gb_batch_set_tuning": (ctypes.c_int, [ctypes.POINTER(GbBatchRule), ctypes.c_int32,
                                           ctypes.POINTER(GbBatchLaunch)]),
    "gb_server_create": (ctypes.c_int, [ctypes.POINTER(GbServerOptions), ctypes.POINTER(ctypes.c_void_p)]),
    "gb_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbColumn), ctypes.c_int32, ctypes.c_int32,
                                        ctypes.POINTER(GbRequest), ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "gb_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(GbQueryInfo)]),
    "gb_server_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(GbOutColumn), ctypes.POINTER(GbOutColumn)]),
    "gb_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "gb_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GbServerStats)]),
    "gb_server_destroy": (None, [ctypes.c_void_p]),
    "gb_aggregate_noalloc": (ctypes.c_int, [ctypes.POINTER(GbColumn), ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(GbRequest), ctypes.c_int32, ctypes.c_int64,
                                            ctypes.POINTER(GbOutColumn), ctypes.POINTER(GbOutColumn),
                                            ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
}


def lib():
    """Loads libcudf_b200.so (raises OSError when it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"cudf_b200 engine library not built: {LIB_PATH} "
                          "(run `python -m cudf_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc == GB_OK:
        return
    msg = (lib().gb_last_error() or b"").decode()
    if rc == GB_ERR_LOGIC:
        raise LogicError(rc, msg)
    if rc == GB_ERR_ALLOC:
        raise MemoryError(msg)
    if rc == GB_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise CudaError(rc, msg)
