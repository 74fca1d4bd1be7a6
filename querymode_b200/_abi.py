"""ctypes mirror of include/qm_gpu.h and the loader for libqm_gpu.so.

The structures here are byte-for-byte the C ABI declared in include/qm_gpu.h;
the product library and the CPU oracle both take them.  Loading the product
library fails loudly when the built .so is missing: there is no CPU fallback
on this path.
"""
from __future__ import annotations

import ctypes as C
import os

# status codes
QM_OK = 0
QM_ERR_INVALID = 1
QM_ERR_UNSUPPORTED = 2
QM_ERR_CUDA = 3
QM_ERR_OOM = 4
QM_ERR_NOT_FOUND = 5
QM_ERR_CAPACITY = 6
QM_ERR_TIMEOUT = 7
QM_ERR_NO_DEVICE = 8
QM_ERR_CANCELLED = 9

STATUS_NAMES = {
    0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CUDA", 4: "OOM", 5: "NOT_FOUND",
    6: "CAPACITY", 7: "TIMEOUT", 8: "NO_DEVICE", 9: "CANCELLED",
}

# dtypes (QMCB tags, src/columnar.ts:22-33) + the result-only 128-bit integer
QM_F64 = 0
QM_PT_SAME, QM_PT_INT8, QM_PT_UINT8, QM_PT_INT16, QM_PT_UINT16, QM_PT_UINT32, QM_PT_FLOAT16 = 0, 1, 2, 3, 4, 5, 6
QM_I64 = 1
QM_I32 = 6
QM_F32 = 7
QM_I128 = 64

# filter ops (src/operators.ts:422-432 codes 0-5)
QM_OP_EQ, QM_OP_NEQ, QM_OP_LT, QM_OP_LTE, QM_OP_GT, QM_OP_GTE = range(6)
QM_OP_BETWEEN = 6
QM_OP_NOT_BETWEEN = 7
QM_OP_IS_NULL = 8
QM_OP_IS_NOT_NULL = 9

OP_CODES = {
    "eq": QM_OP_EQ, "neq": QM_OP_NEQ, "lt": QM_OP_LT, "lte": QM_OP_LTE,
    "gt": QM_OP_GT, "gte": QM_OP_GTE, "between": QM_OP_BETWEEN,
    "not_between": QM_OP_NOT_BETWEEN, "is_null": QM_OP_IS_NULL,
    "is_not_null": QM_OP_IS_NOT_NULL,
}

QM_VAL_NUMBER = 0
QM_VAL_BIGINT = 1

QM_AGG_SUM, QM_AGG_AVG, QM_AGG_MIN, QM_AGG_MAX, QM_AGG_COUNT = range(5)
AGG_CODES = {"sum": QM_AGG_SUM, "avg": QM_AGG_AVG, "min": QM_AGG_MIN,
             "max": QM_AGG_MAX, "count": QM_AGG_COUNT}

QM_NOALLOC_SCRATCH_BYTES = 32 << 20

QM_FLAG_UNORDERED = 1
QM_FLAG_WASM_SCAN_SEMANTICS = 2
QM_FLAG_DETERMINISTIC = 4


class QmColumn(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int32), ("on_device", C.c_int32),
                ("data", C.c_void_p), ("null_bitmap", C.c_void_p)]


class QmValue(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("num", C.c_double),
                ("big", C.c_int64)]


class QmFilter(C.Structure):
    _fields_ = [("column", C.c_char_p), ("op", C.c_int32), ("reserved", C.c_int32),
                ("value", QmValue), ("value2", QmValue)]


class QmAggregate(C.Structure):
    _fields_ = [("fn", C.c_int32), ("reserved", C.c_int32), ("column", C.c_char_p),
                ("alias", C.c_char_p)]


class QmQuery(C.Structure):
    _fields_ = [("filters", C.POINTER(QmFilter)), ("n_filters", C.c_int32),
                ("n_or_groups", C.c_int32), ("or_group_sizes", C.POINTER(C.c_int32)),
                ("or_filters", C.POINTER(QmFilter)), ("group_by", C.POINTER(C.c_char_p)),
                ("n_group_by", C.c_int32), ("n_aggregates", C.c_int32),
                ("aggregates", C.POINTER(QmAggregate)), ("flags", C.c_int32),
                ("reserved", C.c_int32), ("order_by", C.c_char_p), ("order_desc", C.c_int32),
                ("has_limit", C.c_int32), ("limit", C.c_int64), ("offset", C.c_int64)]


class QmTuning(C.Structure):
    _fields_ = [("local_slots", C.c_int32), ("dedupe", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("stage_depth", C.c_int32), ("partitioned", C.c_int32), ("reserved", C.c_int32)]


class QmResultCol(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int32), ("is_key", C.c_int32),
                ("n_rows", C.c_int64), ("data", C.c_void_p), ("null_bitmap", C.c_void_p)]


class QmStats(C.Structure):
    _fields_ = [("rows_scanned", C.c_int64), ("rows_selected", C.c_int64),
                ("groups", C.c_int64), ("bytes_scanned", C.c_int64),
                ("device_ms", C.c_double), ("strategy", C.c_int32),
                ("table_capacity", C.c_int32), ("retries", C.c_int32),
                ("launches", C.c_int32), ("scan_ms", C.c_double)]


class QmServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_batch", C.c_int32), ("max_wait_us", C.c_int32),
                ("max_batch_rows", C.c_int64), ("lanes", C.c_int32), ("max_batch_groups", C.c_int32)]


class QmServerTiming(C.Structure):
    _fields_ = [("queued_us", C.c_int64), ("run_us", C.c_int64), ("total_us", C.c_int64),
                ("batch_size", C.c_int32), ("plan_us", C.c_int32)]


class QmServerCounters(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("cancelled", C.c_int64), ("refused", C.c_int64), ("batches", C.c_int64),
                ("resident_bytes", C.c_int64), ("peak_working_bytes", C.c_int64), ("queued", C.c_int64),
                ("peak_in_flight", C.c_int64), ("heavy", C.c_int64), ("lanes", C.c_int64)]


class QmParquetColumn(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int32), ("reserved", C.c_int32),
                ("chunk", C.c_void_p), ("chunk_bytes", C.c_int64), ("num_values", C.c_int64)]


class QmPage(C.Structure):
    _fields_ = [("buf", C.c_void_p), ("bytes", C.c_int64), ("row_count", C.c_int64), ("null_count", C.c_int64),
                ("data_offset", C.c_int64), ("parquet", C.c_int32), ("reserved", C.c_int32)]


class QmPageColumn(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int32), ("n_pages", C.c_int32), ("pages", C.POINTER(QmPage)),
                ("page_type", C.c_int32), ("reserved", C.c_int32)]


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libqm_gpu.so")

# (name, restype, argtypes) for every entry point of include/qm_gpu.h
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
SIGNATURES = [
    ("qm_version", C.c_char_p, []),
    ("qm_ctx_create", C.c_int, [C.c_int32, _PP]),
    ("qm_ctx_destroy", C.c_int, [_P]),
    ("qm_ctx_last_error", C.c_char_p, [_P]),
    ("qm_ctx_set_stream", C.c_int, [_P, C.c_void_p]),
    ("qm_ctx_trim", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("qm_ctx_set_tuning", C.c_int, [_P, C.c_void_p]),
    ("qm_ctx_device_info", C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    ("qm_table_create", C.c_int, [_P, C.c_int64, C.c_int32, C.POINTER(QmColumn), _PP]),
    ("qm_table_from_qmcb", C.c_int, [_P, C.c_void_p, C.c_size_t, _PP]),
    ("qm_table_destroy", C.c_int, [_P]),
    ("qm_table_num_rows", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("qm_query_run", C.c_int, [_P, _P, C.POINTER(QmQuery), _PP]),
    ("qm_agg_begin", C.c_int, [_P, C.POINTER(QmQuery), _PP]),
    ("qm_agg_push", C.c_int, [_P, C.c_int64, C.c_int32, C.POINTER(QmColumn),
                              C.POINTER(C.c_uint32), C.c_int64]),
    ("qm_agg_finish", C.c_int, [_P, _PP]),
    ("qm_agg_destroy", C.c_int, [_P]),
    ("qm_agg_push_table", C.c_int, [_P, _P]),
    ("qm_agg_partial_export", C.c_int, [_P, C.c_int64, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int32)]),
    ("qm_agg_partial_merge", C.c_int, [_P, C.c_void_p, C.c_int64, C.c_int32, C.c_int64]),
    ("qm_agg_partial_layout", C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("qm_agg_partial_begin", C.c_int, [_P, _PP]),
    ("qm_partial_partition", C.c_int, [_P, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p,
                                       C.POINTER(C.c_int64)]),
    ("qm_filter_select", C.c_int, [_P, C.c_int64, C.c_int32, C.POINTER(QmColumn),
                                   C.POINTER(QmQuery), C.POINTER(C.c_uint32), C.c_int64,
                                   C.POINTER(C.c_uint32), C.c_int64, C.POINTER(C.c_int64)]),
    ("qm_query_run_noalloc", C.c_int, [_P, C.c_int64, C.c_int32, C.POINTER(QmColumn), C.POINTER(QmQuery),
                                       C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    ("qm_batch_create", C.c_int, [_P, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.POINTER(QmQuery)), _PP]),
    ("qm_batch_run", C.c_int, [_P, C.POINTER(C.c_void_p)]),
    ("qm_batch_set_tuning", C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    ("qm_batch_set_mode", C.c_int, [_P, C.c_int32]),
    ("qm_batch_set_waves", C.c_int, [_P, C.c_int32]),
    ("qm_batch_stats", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32)]),
    ("qm_batch_destroy", C.c_int, [_P]),
    ("qm_table_num_columns", C.c_int, [_P, C.POINTER(C.c_int32)]),
    ("qm_table_column", C.c_int, [_P, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_int32)]),
    ("qm_table_from_parquet", C.c_int, [_P, C.c_int32, C.POINTER(QmParquetColumn), _PP]),
    ("qm_table_from_pages", C.c_int, [_P, C.c_int32, C.POINTER(QmPageColumn), _PP]),
    ("qm_table_read_column", C.c_int, [_P, C.c_int32, C.c_void_p, C.c_void_p]),
    ("qm_server_create", C.c_int, [_P, C.POINTER(QmServerConfig), _PP]),
    ("qm_server_submit", C.c_int, [_P, _P, C.POINTER(QmQuery), C.POINTER(C.c_uint64)]),
    ("qm_server_cancel", C.c_int, [_P, C.c_uint64]),
    ("qm_server_wait", C.c_int, [_P, C.c_uint64, C.c_int64, _PP, C.POINTER(QmServerTiming), C.c_char_p,
                                 C.c_size_t]),
    ("qm_server_stats", C.c_int, [_P, C.POINTER(QmServerCounters)]),
    ("qm_server_destroy", C.c_int, [_P]),
    ("qm_result_num_rows", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("qm_result_num_columns", C.c_int, [_P, C.POINTER(C.c_int32)]),
    ("qm_result_column", C.c_int, [_P, C.c_int32, C.POINTER(QmResultCol)]),
    ("qm_result_stats", C.c_int, [_P, C.POINTER(QmStats)]),
    ("qm_result_qmcb", C.c_int, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("qm_result_destroy", C.c_int, [_P]),
]

_lib = None


class QmError(RuntimeError):
    """A non-OK status from the C ABI, with the context's last-error text."""

    def __init__(self, status: int, message: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"QM_ERR_{name}: {message}" if message else f"QM_ERR_{name}")


def load_library(path: str | None = None) -> C.CDLL:
    """Load libqm_gpu.so (built in-tree).  Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libqm_gpu.so not found at {p}; build it with "
            "`python -m querymode_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
