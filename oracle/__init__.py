"""CPU oracle for the filter -> GROUP BY path — TEST INFRASTRUCTURE ONLY.

This package is the parity checker for the CUDA path and the timed CPU
baseline.  It is imported only by tests/, bench.py's CPU-baseline and
reference arms, and __graft_entry__.smoke(); the product package never
imports or calls it.

`liboracle.so` (built from qm_oracle.c by oracle/Makefile) restates the
reference's semantics; see the header of qm_oracle.c for the file:line map.
`jsref.py` is a second, literal restatement in pure Python (string group
keys, Map first-seen order) for small inputs, used to pin the C oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from querymode_b200 import _abi as A
from querymode_b200.engine import Result, ResultColumn, _ColumnSet, _read_col
from querymode_b200.query import CQuery, QueryDescriptor

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "qm_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(src) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "all"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [C.c_int64, C.c_int32, C.POINTER(A.QmColumn), C.POINTER(A.QmQuery),
                                 C.c_int64, C.POINTER(P)]
        L.oracle_run_mt.restype = C.c_int
        L.oracle_run_mt.argtypes = [C.c_int64, C.c_int32, C.POINTER(A.QmColumn), C.POINTER(A.QmQuery),
                                    C.c_int64, C.c_int32, C.POINTER(P)]
        L.oracle_run_keypart.restype = C.c_int
        L.oracle_run_keypart.argtypes = [C.c_int64, C.c_int32, C.POINTER(A.QmColumn), C.POINTER(A.QmQuery),
                                         C.c_int32, C.POINTER(P)]
        L.oracle_filter_select.restype = C.c_int
        L.oracle_filter_select.argtypes = [C.c_int64, C.c_int32, C.POINTER(A.QmColumn),
                                           C.POINTER(A.QmQuery), C.POINTER(C.c_uint32), C.c_int64,
                                           C.POINTER(C.c_int64)]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_result_num_rows.restype = C.c_int64
        L.oracle_result_num_rows.argtypes = [P]
        L.oracle_result_num_columns.restype = C.c_int32
        L.oracle_result_num_columns.argtypes = [P]
        L.oracle_result_column.restype = C.c_int
        L.oracle_result_column.argtypes = [P, C.c_int32, C.POINTER(A.QmResultCol)]
        L.oracle_result_diag.restype = C.c_int
        L.oracle_result_diag.argtypes = [P, C.c_int32, C.POINTER(C.POINTER(C.c_double)),
                                         C.POINTER(C.POINTER(C.c_double)),
                                         C.POINTER(C.POINTER(C.c_double))]
        L.oracle_result_destroy.restype = None
        L.oracle_result_destroy.argtypes = [P]
        _lib = L
    return _lib


class OracleResult(Result):
    """Result plus, per float SUM/AVG column, the 113-bit sum and sum of
    magnitudes of every group (for the 1e-12 tolerance checks)."""

    def __init__(self, columns, n_rows, diag):
        super().__init__(columns, n_rows)
        self.diag = diag  # name -> (exact_sum float64 pair summed, abs_sum)

    def take(self, order) -> "OracleResult":
        idx = np.asarray(order, dtype=np.int64)
        base = Result.take(self, idx)
        return OracleResult(base.columns, base.n_rows, {k: tuple(a[idx] for a in v) for k, v in self.diag.items()})


def _collect(L, h) -> OracleResult:
    n = L.oracle_result_num_rows(h)
    nc = L.oracle_result_num_columns(h)
    cols, diag = [], {}
    for i in range(nc):
        rc = A.QmResultCol()
        L.oracle_result_column(h, i, C.byref(rc))
        col = _read_col(rc, n)
        cols.append(col)
        hi = C.POINTER(C.c_double)()
        lo = C.POINTER(C.c_double)()
        ab = C.POINTER(C.c_double)()
        L.oracle_result_diag(h, i, C.byref(hi), C.byref(lo), C.byref(ab))
        if hi and n:
            diag[col.name] = (np.ctypeslib.as_array(hi, (n,)).copy(),
                              np.ctypeslib.as_array(lo, (n,)).copy(),
                              np.ctypeslib.as_array(ab, (n,)).copy())
    return OracleResult(cols, n, diag)


def run(columns, query: QueryDescriptor, batch_rows: int = 0, threads: int = 1) -> OracleResult:
    """The reference's result for `query` over `columns` (numpy arrays or
    engine.Column), aggregated in batches of `batch_rows` rows (0: one batch)."""
    L = lib()
    cs = _ColumnSet(columns)
    cq = CQuery(query)
    h = C.c_void_p()
    if threads <= 1:
        st = L.oracle_run(cs.n_rows, cs.count, cs.array, cq.ref, batch_rows, C.byref(h))
    else:
        st = L.oracle_run_mt(cs.n_rows, cs.count, cs.array, cq.ref, batch_rows, threads, C.byref(h))
    if st != 0:
        raise A.QmError(st, L.oracle_last_error().decode())
    try:
        return _collect(L, h)
    finally:
        L.oracle_result_destroy(h)


def run_full(columns, query: QueryDescriptor, threads: int | None = None) -> OracleResult:
    """The reference's one-batch result (run(..., batch_rows=0)) bit for bit,
    on `threads` host threads (default: all): groups are split across threads
    by key hash, each group's rows visited in row order, and the groups put
    back in first-seen order.  For full-size checks of large tables."""
    L = lib()
    cs = _ColumnSet(columns)
    cq = CQuery(query)
    h = C.c_void_p()
    st = L.oracle_run_keypart(cs.n_rows, cs.count, cs.array, cq.ref, threads or os.cpu_count() or 1, C.byref(h))
    if st != 0:
        raise A.QmError(st, L.oracle_last_error().decode())
    try:
        return _collect(L, h)
    finally:
        L.oracle_result_destroy(h)


def filter_select(columns, query: QueryDescriptor, selection=None) -> np.ndarray:
    if selection is not None:
        sel = np.asarray(selection, dtype=np.int64)
        sub = {}
        for k, v in columns.items():
            if hasattr(v, "values"):
                sub[k] = type(v)(np.asarray(v.values)[sel], None if v.nulls is None else np.asarray(v.nulls)[sel])
            else:
                sub[k] = np.asarray(v)[sel]
        return sel[filter_select(sub, query)].astype(np.uint32)
    L = lib()
    cs = _ColumnSet(columns)
    cq = CQuery(query)
    out = np.empty(max(cs.n_rows, 1), dtype=np.uint32)
    cnt = C.c_int64()
    st = L.oracle_filter_select(cs.n_rows, cs.count, cs.array, cq.ref,
                                out.ctypes.data_as(C.POINTER(C.c_uint32)), cs.n_rows, C.byref(cnt))
    if st != 0:
        raise A.QmError(st, L.oracle_last_error().decode())
    return out[:cnt.value].copy()


__all__ = ["run", "run_full", "filter_select", "build", "OracleResult", "ResultColumn"]
