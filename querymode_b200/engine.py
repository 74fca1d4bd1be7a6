"""Host-side handles over the C ABI: Context, Table, Result, AggStream.

Everything here calls libqm_gpu.so through ctypes; there is no CPU compute
path.  Columns are numpy arrays (int32 / int64 / float32 / float64) with an
optional boolean NULL mask, or torch CUDA tensors already resident in HBM
(passed by device pointer, read in place).
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass
from typing import Any, Mapping

import numpy as np

from . import _abi as A
from .query import CQuery, QueryDescriptor

_NP_DTYPES = {
    np.dtype(np.int32): A.QM_I32,
    np.dtype(np.int64): A.QM_I64,
    np.dtype(np.float32): A.QM_F32,
    np.dtype(np.float64): A.QM_F64,
}
_QM_TO_NP = {A.QM_I32: np.int32, A.QM_I64: np.int64, A.QM_F32: np.float32, A.QM_F64: np.float64}


def _check(lib, ctx_ptr, status: int) -> None:
    if status != A.QM_OK:
        msg = lib.qm_ctx_last_error(ctx_ptr) if ctx_ptr else b""
        raise A.QmError(status, (msg or b"").decode(errors="replace"))


def pack_nulls(mask: np.ndarray | None) -> np.ndarray | None:
    """Boolean NULL mask -> QMCB bitmap (bit set = NULL, LSB first)."""
    if mask is None:
        return None
    mask = np.asarray(mask, dtype=bool)
    if not mask.any():
        return None
    return np.packbits(mask, bitorder="little")


def unpack_nulls(bits: np.ndarray, n: int) -> np.ndarray:
    return np.unpackbits(bits, count=n, bitorder="little").astype(bool)


@dataclass
class Column:
    """One input column: values plus an optional NULL mask (True = NULL)."""
    values: Any
    nulls: np.ndarray | None = None


@dataclass
class Page:
    """One page buffer of a scan (the reference's PageInfo beside its bytes):
    `buf` any bytes-like object or uint8 array (read in place, not copied);
    `parquet` marks a Parquet column chunk of `row_count` values (PageInfo
    with an encoding); otherwise a PLAIN page with an optional validity
    bitmap, `data_offset` = PageInfo.dataOffsetInPage."""
    buf: Any
    row_count: int = 0
    null_count: int = 0
    data_offset: int | None = None
    parquet: bool = False


@dataclass
class PageTable:
    """A column's pages as a reader has them: one host buffer holding the
    page bytes (a column's byte range of a file) and per page its offset and
    length in it (PageInfo.byteOffset / byteLength), rowCount, nullCount and,
    optionally, dataOffsetInPage (-1 = absent) and the Parquet flag."""
    buf: Any
    offsets: np.ndarray
    lengths: np.ndarray
    row_counts: np.ndarray
    null_counts: np.ndarray | None = None
    data_offsets: np.ndarray | None = None
    parquet: np.ndarray | None = None


# numpy image of qm_page (checked against the ctypes mirror at import)
_PAGE_DTYPE = np.dtype([("buf", np.uint64), ("bytes", np.int64), ("row_count", np.int64), ("null_count", np.int64),
                        ("data_offset", np.int64), ("parquet", np.int32), ("reserved", np.int32)])
assert _PAGE_DTYPE.itemsize == C.sizeof(A.QmPage) and all(
    _PAGE_DTYPE.fields[f][1] == getattr(A.QmPage, f).offset for f, _ in A.QmPage._fields_)


def _page_records(pages) -> tuple[np.ndarray, list]:
    """qm_page records of a PageTable or a list of Page, and the objects that
    must stay alive while they are used."""
    if isinstance(pages, PageTable):
        b = _host_bytes(pages.buf)
        n = len(pages.offsets)
        offs = np.asarray(pages.offsets, dtype=np.int64)
        lens = np.asarray(pages.lengths, dtype=np.int64)
        if n and (offs.min() < 0 or (offs + lens).max() > b.nbytes or lens.min() < 0):
            raise ValueError("page ranges outside the buffer")
        rec = np.zeros(n, dtype=_PAGE_DTYPE)
        rec["buf"] = np.uint64(b.ctypes.data) + offs.astype(np.uint64)
        rec["bytes"] = lens
        rec["row_count"] = pages.row_counts
        rec["null_count"] = 0 if pages.null_counts is None else pages.null_counts
        rec["data_offset"] = -1 if pages.data_offsets is None else pages.data_offsets
        rec["parquet"] = 0 if pages.parquet is None else pages.parquet
        return rec, [b]
    rec = np.zeros(len(pages), dtype=_PAGE_DTYPE)
    keep = []
    for k, pg in enumerate(pages):
        b = _host_bytes(pg.buf)
        keep.append(b)
        rec[k] = (b.__array_interface__["data"][0] if b.nbytes else 0, b.nbytes, pg.row_count, pg.null_count,
                  -1 if pg.data_offset is None else pg.data_offset, 1 if pg.parquet else 0, 0)
    return rec, keep


def _host_bytes(obj) -> np.ndarray:
    a = obj if isinstance(obj, np.ndarray) else np.frombuffer(obj, dtype=np.uint8)
    if not a.flags.c_contiguous:
        raise ValueError("page buffers must be contiguous")
    return a


class _ColumnSet:
    """Builds the qm_column array for a mapping of name -> array / Column and
    keeps every referenced buffer alive while the C side may read it."""

    def __init__(self, columns: Mapping[str, Any]):
        self.keep: list = []
        cols = []
        n_rows = None
        for name, v in columns.items():
            nulls = None
            if isinstance(v, Column):
                v, nulls = v.values, v.nulls
            c = A.QmColumn()
            nm = name.encode()
            self.keep.append(nm)
            c.name = nm
            if _is_torch_cuda(v):
                import torch  # noqa: F401  (plumbing for device-resident input)
                if not v.is_contiguous():
                    v = v.contiguous()
                dt = _torch_dtype(v)
                c.dtype = dt
                c.on_device = 1
                c.data = v.data_ptr()
                n = v.numel()
                self.keep.append(v)
                if nulls is not None:
                    raise ValueError("device-resident columns take no host NULL mask")
            else:
                arr = np.ascontiguousarray(v)
                if arr.dtype not in _NP_DTYPES:
                    raise TypeError(f"column {name}: dtype {arr.dtype} is not on the GPU path")
                c.dtype = _NP_DTYPES[arr.dtype]
                c.on_device = 0
                c.data = arr.ctypes.data if arr.size else None
                n = arr.size
                self.keep.append(arr)
                nb = pack_nulls(nulls)
                if nb is not None:
                    if len(nulls) != n:
                        raise ValueError(f"column {name}: NULL mask length {len(nulls)} != {n}")
                    self.keep.append(nb)
                    c.null_bitmap = nb.ctypes.data
            if n_rows is None:
                n_rows = n
            elif n != n_rows:
                raise ValueError(f"column {name} has {n} rows, expected {n_rows}")
            cols.append(c)
        self.n_rows = n_rows or 0
        self.array = (A.QmColumn * max(1, len(cols)))(*cols)
        self.count = len(cols)


def _is_torch_cuda(v) -> bool:
    mod = type(v).__module__
    return mod.startswith("torch") and getattr(v, "is_cuda", False)


def _torch_dtype(t) -> int:
    import torch
    m = {torch.int32: A.QM_I32, torch.int64: A.QM_I64, torch.float32: A.QM_F32,
         torch.float64: A.QM_F64}
    if t.dtype not in m:
        raise TypeError(f"tensor dtype {t.dtype} is not on the GPU path")
    return m[t.dtype]


@dataclass
class ResultColumn:
    name: str
    dtype: int
    is_key: bool
    values: np.ndarray       # I128 columns: shape (n, 2) int64 [lo, hi]
    nulls: np.ndarray | None  # bool, True = NULL

    def pyvalues(self) -> list:
        """Python values: int for integer results, float for float ones,
        None for NULL."""
        n = len(self.values)
        if self.dtype == A.QM_I128:
            lo = self.values[:, 0].astype(np.uint64)
            hi = self.values[:, 1]
            out = [(int(h) << 64) | int(l) for l, h in zip(lo, hi)]
        elif self.dtype == A.QM_F64:
            out = [float(x) for x in self.values]
        else:
            out = [int(x) for x in self.values]
        if self.nulls is not None:
            out = [None if self.nulls[i] else out[i] for i in range(n)]
        return out


@dataclass
class Stats:
    rows_scanned: int
    rows_selected: int
    groups: int
    bytes_scanned: int
    device_ms: float
    strategy: int
    table_capacity: int
    retries: int
    launches: int
    scan_ms: float


class Result:
    """Typed result columns (keys first, then aggregates in query order)."""

    def __init__(self, columns: list[ResultColumn] | None, n_rows: int, stats: Stats | None = None,
                 qmcb: bytes | None = None, build=None):
        self._columns = columns
        self._build = build  # makes the columns on first use (views of a result handle)
        self.n_rows = n_rows
        self.stats = stats
        self.qmcb = qmcb

    @property
    def columns(self) -> list[ResultColumn]:
        if self._columns is None:
            self._columns = self._build()
            self._build = None
        return self._columns

    @columns.setter
    def columns(self, cols: list[ResultColumn]) -> None:
        self._columns = cols
        self._build = None

    def take(self, order) -> "Result":
        """The rows at `order` (a list of row indices), as a new Result."""
        idx = np.asarray(order, dtype=np.int64)
        cols = [ResultColumn(c.name, c.dtype, c.is_key, c.values[idx],
                             None if c.nulls is None else c.nulls[idx]) for c in self.columns]
        return Result(cols, len(idx), self.stats)

    def column(self, name: str) -> ResultColumn:
        for c in self.columns:
            if c.name == name:
                return c
        raise KeyError(name)

    @property
    def names(self) -> list[str]:
        return [c.name for c in self.columns]

    @classmethod
    def from_handle(cls, lib, handle: C.c_void_p, with_qmcb: bool = False, owned: bool = False) -> "Result":
        """Wrap a qm_result.  With owned=True the columns are zero-copy views of
        the result's pinned host buffer and the handle is destroyed when the
        last view goes away; otherwise the columns are copies."""
        n = C.c_int64()
        nc = C.c_int32()
        lib.qm_result_num_rows(handle, C.byref(n))
        lib.qm_result_num_columns(handle, C.byref(nc))
        owner = _ResultOwner(lib, handle) if owned else None

        def build():
            cols = []
            for i in range(nc.value):
                rc = A.QmResultCol()
                lib.qm_result_column(handle, i, C.byref(rc))
                cols.append(_view_col(rc, n.value, owner) if owned else _read_col(rc, n.value))
            return cols

        # owned results keep their handle (through `owner`) until the columns
        # are made and dropped; copies are made now, before the handle goes
        cols = None if owned else build()
        st = A.QmStats()
        lib.qm_result_stats(handle, C.byref(st))
        stats = Stats(st.rows_scanned, st.rows_selected, st.groups, st.bytes_scanned, st.device_ms,
                      st.strategy, st.table_capacity, st.retries, st.launches, st.scan_ms)
        qmcb = None
        if with_qmcb:
            p = C.c_void_p()
            ln = C.c_size_t()
            if lib.qm_result_qmcb(handle, C.byref(p), C.byref(ln)) == A.QM_OK:
                qmcb = C.string_at(p, ln.value)
        if owned:
            keep = owner  # the handle lives as long as the result may still build views of it
            return cls(None, n.value, stats, qmcb, build=lambda: (keep, build())[1])
        return cls(cols, n.value, stats, qmcb)


class _ResultOwner:
    """Destroys a qm_result once no numpy view of its buffer is alive."""

    def __init__(self, lib, handle):
        self.lib = lib
        self.handle = C.c_void_p(handle.value if isinstance(handle, C.c_void_p) else handle)

    def __del__(self):
        try:
            if self.handle:
                self.lib.qm_result_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def _buffer_view(addr: int, nbytes: int, owner: _ResultOwner) -> np.ndarray:
    buf = (C.c_uint8 * max(nbytes, 1)).from_address(addr)
    buf._owner = owner  # the ctypes array keeps the result alive; numpy keeps the array
    return np.frombuffer(buf, dtype=np.uint8, count=nbytes)


def _view_col(rc: A.QmResultCol, n: int, owner: _ResultOwner) -> ResultColumn:
    name = rc.name.decode()
    if n == 0 or not rc.data:
        return _read_col(rc, n)
    if rc.dtype == A.QM_I128:
        vals = _buffer_view(rc.data, 16 * n, owner).view(np.int64).reshape(n, 2)
    else:
        dt = np.dtype(_QM_TO_NP[rc.dtype])
        vals = _buffer_view(rc.data, dt.itemsize * n, owner).view(dt)
    nulls = None
    if rc.null_bitmap:
        bits = _buffer_view(rc.null_bitmap, (n + 7) // 8, owner)
        nulls = unpack_nulls(bits, n)
    return ResultColumn(name, rc.dtype, bool(rc.is_key), vals, nulls)


def _read_col(rc: A.QmResultCol, n: int) -> ResultColumn:
    name = rc.name.decode()
    if rc.dtype == A.QM_I128:
        buf = C.string_at(rc.data, 16 * n) if n else b""
        vals = np.frombuffer(buf, dtype=np.int64).reshape(n, 2).copy()
    else:
        dt = _QM_TO_NP[rc.dtype]
        size = np.dtype(dt).itemsize
        buf = C.string_at(rc.data, size * n) if n else b""
        vals = np.frombuffer(buf, dtype=dt).copy()
    nulls = None
    if rc.null_bitmap:
        bits = np.frombuffer(C.string_at(rc.null_bitmap, (n + 7) // 8), dtype=np.uint8)
        nulls = unpack_nulls(bits, n)
    return ResultColumn(name, rc.dtype, bool(rc.is_key), vals, nulls)


class Context:
    """A qm_ctx: one CUDA device, one stream, cached scratch memory.

    Like the reference's per-Durable-Object engine, a context serves one host
    thread at a time."""

    def __init__(self, device: int = 0, lib: C.CDLL | None = None):
        self.lib = lib or A.load_library()
        h = C.c_void_p()
        st = self.lib.qm_ctx_create(device, C.byref(h))
        if st != A.QM_OK:
            raise A.QmError(st, f"qm_ctx_create(device={device})")
        self.h = h
        self.device = device
        self._children = weakref.WeakSet()

    def _adopt(self, child) -> None:
        """Track a table / batch / stream / server made on this context: the
        context closes them before itself, whatever order they are collected
        in."""
        self._children.add(child)

    def close(self) -> None:
        if getattr(self, "h", None):
            for child in sorted(list(self._children), key=lambda c: c._close_order):
                child.close()
            self.lib.qm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, status: int) -> None:
        _check(self.lib, self.h, status)

    def set_stream(self, stream_handle: int | None) -> None:
        """Order this context's work on a CUDA stream handle (e.g.
        ``torch.cuda.current_stream().cuda_stream``); None restores the
        context's own stream."""
        self.check(self.lib.qm_ctx_set_stream(self.h, stream_handle or None))

    def trim(self) -> int:
        """Free the device blocks kept from destroyed tables; returns the
        bytes freed."""
        n = C.c_int64()
        self.check(self.lib.qm_ctx_trim(self.h, C.byref(n)))
        return n.value

    def set_tuning(self, local_slots: int = 0, dedupe: int = -1, blocks_per_sm: int = 0,
                   stage_depth: int = 0, partitioned: int = 0) -> None:
        """Launch-shape knobs of the fused scan (see qm_tuning); the
        defaults restore the planner's choices."""
        t = A.QmTuning(local_slots, dedupe, blocks_per_sm, stage_depth, partitioned)
        self._tuning = t
        self.check(self.lib.qm_ctx_set_tuning(self.h, C.byref(t)))

    def device_info(self) -> tuple[int, int]:
        sm = C.c_int32()
        hbm = C.c_int64()
        self.check(self.lib.qm_ctx_device_info(self.h, C.byref(sm), C.byref(hbm)))
        return sm.value, hbm.value

    # -- tables --------------------------------------------------------------
    def table(self, columns: Mapping[str, Any]) -> "Table":
        cs = _ColumnSet(columns)
        h = C.c_void_p()
        self.check(self.lib.qm_table_create(self.h, cs.n_rows, cs.count, cs.array, C.byref(h)))
        return Table(self, h, cs.n_rows, list(columns.keys()), keep=cs.keep)

    def table_from_parquet_chunks(self, chunks: list[tuple[str, int, bytes, int]]) -> "Table":
        """A table from Parquet column chunks (name, QM dtype, chunk bytes
        from the first page header, ColumnMetaData.num_values), PLAIN pages
        decoded on the device."""
        n = len(chunks)
        arr = (A.QmParquetColumn * n)()
        keep = []
        for i, (name, dtype, data, num_values) in enumerate(chunks):
            nb = name.encode()
            buf = C.create_string_buffer(bytes(data), len(data))
            keep += [nb, buf]
            arr[i].name = nb
            arr[i].dtype = dtype
            arr[i].chunk = C.cast(buf, C.c_void_p)
            arr[i].chunk_bytes = len(data)
            arr[i].num_values = num_values
        h = C.c_void_p()
        self.check(self.lib.qm_table_from_parquet(self.h, n, arr, C.byref(h)))
        rows = C.c_int64()
        self.check(self.lib.qm_table_num_rows(h, C.byref(rows)))
        t = Table(self, h, rows.value, [c[0] for c in chunks])
        t._dtypes = [c[1] for c in chunks]
        return t

    def table_from_pages(self, columns: list[tuple]) -> "Table":
        """A table from scan pages: per column (name, QM dtype, its pages in
        order as a list of Page or a PageTable[, QM_PT_* page value type]),
        decoded on the device and concatenated page after page.  Pages of a
        narrower type (int8 / uint8 / int16 / uint16 into QM_I32, uint32 into
        QM_F64, float16 into QM_F32) are widened as the reference's numbers
        hold them."""
        n = len(columns)
        arr = (A.QmPageColumn * n)()
        keep = []
        for i, col in enumerate(columns):
            name, dtype, pages = col[:3]
            arr[i].page_type = col[3] if len(col) > 3 else A.QM_PT_SAME
            nb = name.encode()
            rec, k = _page_records(pages)
            keep += [nb, rec, k]
            arr[i].name = nb
            arr[i].dtype = dtype
            arr[i].n_pages = len(rec)
            arr[i].pages = rec.ctypes.data_as(C.POINTER(A.QmPage))
        h = C.c_void_p()
        self.check(self.lib.qm_table_from_pages(self.h, n, arr, C.byref(h)))
        rows = C.c_int64()
        self.check(self.lib.qm_table_num_rows(h, C.byref(rows)))
        t = Table(self, h, rows.value, [c[0] for c in columns])
        t._dtypes = [c[1] for c in columns]
        return t

    def table_from_parquet(self, path: str, row_group: int = 0, columns: list[str] | None = None) -> "Table":
        """One row group of a Parquet file: its INT32 / INT64 / FLOAT / DOUBLE
        columns (or `columns`), located through the file's footer (pyarrow
        reads the footer only; the pages are decoded on the device)."""
        import pyarrow.parquet as pq
        types = {"INT32": A.QM_I32, "INT64": A.QM_I64, "FLOAT": A.QM_F32, "DOUBLE": A.QM_F64}
        md = pq.ParquetFile(path).metadata.row_group(row_group)
        with open(path, "rb") as f:
            raw = f.read()
        chunks = []
        for c in range(md.num_columns):
            cc = md.column(c)
            name = cc.path_in_schema
            if columns is not None and name not in columns:
                continue
            if cc.physical_type not in types:
                if columns is not None:
                    raise ValueError(f"column {name}: {cc.physical_type} is not a numeric column")
                continue
            start = cc.dictionary_page_offset if cc.dictionary_page_offset is not None else cc.data_page_offset
            chunks.append((name, types[cc.physical_type], raw[start:start + cc.total_compressed_size],
                           cc.num_values))
        return self.table_from_parquet_chunks(chunks)

    def table_from_qmcb(self, buf: bytes) -> "Table":
        b = bytes(buf)
        h = C.c_void_p()
        self.check(self.lib.qm_table_from_qmcb(self.h, b, len(b), C.byref(h)))
        n = C.c_int64()
        self.lib.qm_table_num_rows(h, C.byref(n))
        k = C.c_int32()
        self.check(self.lib.qm_table_num_columns(h, C.byref(k)))
        names, dtypes = [], []
        for i in range(k.value):
            nm, dt = C.c_char_p(), C.c_int32()
            self.check(self.lib.qm_table_column(h, i, C.byref(nm), C.byref(dt)))
            names.append(nm.value.decode("utf-8", "replace"))
            dtypes.append(dt.value)
        t = Table(self, h, n.value, names)
        t._dtypes = dtypes
        return t

    # -- filter-only ---------------------------------------------------------
    def filter_select(self, columns: Mapping[str, Any], query: QueryDescriptor,
                      selection: np.ndarray | None = None) -> np.ndarray:
        """Ascending indices of the rows (of `selection`, if given) passing
        query's filters."""
        cs = _ColumnSet(columns)
        cq = CQuery(query)
        sel_ptr, n_sel = None, 0
        if selection is not None:
            sel = np.ascontiguousarray(selection, dtype=np.uint32)
            cs.keep.append(sel)
            sel_ptr = sel.ctypes.data_as(C.POINTER(C.c_uint32))
            n_sel = sel.size
        cap = n_sel if selection is not None else cs.n_rows
        out = np.empty(max(cap, 1), dtype=np.uint32)
        cnt = C.c_int64()
        self.check(self.lib.qm_filter_select(
            self.h, cs.n_rows, cs.count, cs.array, cq.ref, sel_ptr, n_sel,
            out.ctypes.data_as(C.POINTER(C.c_uint32)), cap, C.byref(cnt)))
        return out[:cnt.value].copy()

    def aggregate(self, query: QueryDescriptor) -> "AggStream":
        return AggStream(self, query)

    def partition_partial(self, rows, parts: int):
        """Partial rows (an int64 CUDA tensor [n, row_words] from
        AggStream.export_partial) split by key hash into `parts` parts:
        (the rows part after part, each part's row count)."""
        import torch
        rows = rows.contiguous()
        out = torch.empty_like(rows)
        counts = (C.c_int64 * parts)()
        torch.cuda.current_stream(rows.device).synchronize()
        self.check(self.lib.qm_partial_partition(self.h, C.c_void_p(rows.data_ptr()) if rows.numel() else None,
                                                 rows.shape[0], rows.shape[1], parts,
                                                 C.c_void_p(out.data_ptr()) if rows.numel() else None, counts))
        return out, [int(c) for c in counts]

    def batch(self, tables: list["Table"], queries: list[QueryDescriptor]) -> "Batch":
        return Batch(self, tables, queries)

    def server(self, hbm_budget_bytes: int, max_batch: int = 64, max_wait_us: int = 0,
               max_batch_rows: int = 0, lanes: int = 0, max_batch_groups: int = 0) -> "Server":
        return Server(self, hbm_budget_bytes, max_batch, max_wait_us, max_batch_rows, lanes, max_batch_groups)


class Table:
    """A qm_table: numeric columns resident in HBM."""

    def __init__(self, ctx: Context, h: C.c_void_p, n_rows: int, names: list[str], keep=None):
        self.ctx = ctx
        self.h = h
        self.n_rows = n_rows
        self.names = names
        self._keep = keep  # device-resident inputs are read in place
        ctx._adopt(self)

    _close_order = 2

    def read_column(self, name: str) -> tuple[np.ndarray, np.ndarray]:
        """A column copied back to the host: (values, NULL mask)."""
        idx = self.names.index(name)
        dtypes = {A.QM_I32: np.int32, A.QM_I64: np.int64, A.QM_F32: np.float32, A.QM_F64: np.float64}
        raw_types = getattr(self, "_dtypes", None)
        if not raw_types:
            raise ValueError("read_column needs a table whose column dtypes are known (table_from_parquet)")
        vals = np.empty(self.n_rows, dtype=dtypes[raw_types[idx]])
        nulls = np.empty(self.n_rows, dtype=np.uint8)
        self.ctx.check(self.ctx.lib.qm_table_read_column(self.h, idx, vals.ctypes.data_as(C.c_void_p),
                                                         nulls.ctypes.data_as(C.c_void_p)))
        return vals, nulls.astype(bool)

    def close(self) -> None:
        if getattr(self, "h", None):
            if self.ctx.h:
                self.ctx.lib.qm_table_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, query: QueryDescriptor | CQuery, with_qmcb: bool = False) -> Result:
        """Run a query; the result's columns are zero-copy views of its
        pinned host buffer.  A CQuery may be passed to skip re-lowering."""
        cq = query if isinstance(query, CQuery) else CQuery(query)
        r = C.c_void_p()
        self.ctx.check(self.ctx.lib.qm_query_run(self.ctx.h, self.h, cq.ref, C.byref(r)))
        return Result.from_handle(self.ctx.lib, r, with_qmcb, owned=True)


class AggStream:
    """Streaming aggregation: push batches in order, then finish
    (AggregateOperator.next's drain loop, src/operators.ts:1656-1681)."""

    def __init__(self, ctx: Context, query: QueryDescriptor):
        self.ctx = ctx
        self.cq = CQuery(query)
        h = C.c_void_p()
        ctx.check(ctx.lib.qm_agg_begin(ctx.h, self.cq.ref, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def push(self, columns: Mapping[str, Any], selection: np.ndarray | None = None) -> None:
        cs = _ColumnSet(columns)
        sel_ptr = None
        n_sel = 0
        if selection is not None:
            sel = np.ascontiguousarray(selection, dtype=np.uint32)
            cs.keep.append(sel)
            sel_ptr = sel.ctypes.data_as(C.POINTER(C.c_uint32))
            n_sel = sel.size
        self.ctx.check(self.ctx.lib.qm_agg_push(self.h, cs.n_rows, cs.count, cs.array, sel_ptr, n_sel))

    def push_table(self, table: "Table") -> None:
        """Push a registered table's rows as one batch (read in place)."""
        self.ctx.check(self.ctx.lib.qm_agg_push_table(self.h, table.h))

    def export_partial(self, row_offset: int = 0):
        """This shard's occupied group slots as partial rows: an int64 CUDA
        tensor [groups, row_words] on the context's device (key word,
        special flag, accumulator words; FIRST moved by row_offset, the
        shard's first global row)."""
        import torch
        n = C.c_int64()
        w = C.c_int32()
        self.ctx.check(self.ctx.lib.qm_agg_partial_export(self.h, row_offset, None, 0, C.byref(n), C.byref(w)))
        out = torch.empty((n.value, w.value), dtype=torch.int64, device=f"cuda:{self.ctx.device}")
        torch.cuda.current_stream(self.ctx.device).synchronize()
        self.ctx.check(self.ctx.lib.qm_agg_partial_export(self.h, row_offset, C.c_void_p(out.data_ptr()),
                                                          n.value, C.byref(n), C.byref(w)))
        return out

    def merge_partial(self, rows, rows_end: int) -> None:
        """Fold another shard's partial rows (a CUDA tensor on this context's
        device, from export_partial) into this aggregation; rows_end bounds
        the global rows they cover."""
        import torch
        rows = rows.contiguous()
        if rows.dtype != torch.int64 or rows.dim() != 2:
            raise ValueError("partial rows are an int64 [groups, row_words] tensor")
        torch.cuda.current_stream(rows.device).synchronize()
        self.ctx.check(self.ctx.lib.qm_agg_partial_merge(self.h, C.c_void_p(rows.data_ptr()) if rows.numel() else None,
                                                         rows.shape[0], rows.shape[1], rows_end))

    def partial_layout(self) -> tuple[int, int]:
        """(words per partial row, word of the group's first global row or -1)."""
        w = C.c_int32()
        f = C.c_int32()
        self.ctx.check(self.ctx.lib.qm_agg_partial_layout(self.h, C.byref(w), C.byref(f)))
        return w.value, f.value

    def partial_begin(self) -> "AggStream":
        """A new empty aggregation with this one's plan, for merging the
        partial rows of one key range (the receiving side of a
        key-partitioned exchange)."""
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.qm_agg_partial_begin(self.h, C.byref(h)))
        other = AggStream.__new__(AggStream)
        other.ctx = self.ctx
        other.cq = self.cq
        other.h = h
        self.ctx._adopt(other)
        return other

    def finish(self, with_qmcb: bool = False) -> Result:
        r = C.c_void_p()
        self.ctx.check(self.ctx.lib.qm_agg_finish(self.h, C.byref(r)))
        try:
            return Result.from_handle(self.ctx.lib, r, with_qmcb)
        finally:
            self.ctx.lib.qm_result_destroy(r)

    _close_order = 1

    def close(self) -> None:
        if getattr(self, "h", None):
            if self.ctx.h:
                self.ctx.lib.qm_agg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A qm_batch: many queries (query i over tables[i]) in one persistent
    fused launch, CUDA-graph captured on the first run."""

    def __init__(self, ctx: Context, tables: list[Table], queries: list[QueryDescriptor]):
        if len(tables) != len(queries):
            raise ValueError("one table per query")
        self.ctx = ctx
        self.tables = tables
        self.cqs = [q if isinstance(q, CQuery) else CQuery(q) for q in queries]
        n = len(queries)
        th = (C.c_void_p * n)(*[t.h.value for t in tables])
        qs = (C.POINTER(A.QmQuery) * n)(*[C.pointer(cq.struct) for cq in self.cqs])
        h = C.c_void_p()
        ctx.check(ctx.lib.qm_batch_create(ctx.h, n, th, qs, C.byref(h)))
        self.h = h
        self.n = n
        ctx._adopt(self)

    def set_tuning(self, chunk_tiles: int = -1, local_kb: int = -1, blocks_per_sm: int = -1) -> None:
        self.ctx.check(self.ctx.lib.qm_batch_set_tuning(self.h, chunk_tiles, local_kb, blocks_per_sm))

    def set_mode(self, mode: int) -> None:
        """1: one specialised scan launch per query on parallel graph
        branches (default); 0: persistent kernels, one per query class."""
        self.ctx.check(self.ctx.lib.qm_batch_set_mode(self.h, mode))

    def set_waves(self, waves: int) -> None:
        """Cut the batch into `waves` waves (0: by batch size), each one's
        results copied to the host while the later waves run."""
        self.ctx.check(self.ctx.lib.qm_batch_set_waves(self.h, waves))

    def run(self) -> "BatchResults":
        out = (C.c_void_p * self.n)()
        self.ctx.check(self.ctx.lib.qm_batch_run(self.h, out))
        return BatchResults(self.ctx.lib, [out[i] for i in range(self.n)])

    def stats(self) -> dict:
        ms = C.c_double()
        rows = C.c_int64()
        nbytes = C.c_int64()
        chunks = C.c_int32()
        self.ctx.check(self.ctx.lib.qm_batch_stats(self.h, C.byref(ms), C.byref(rows), C.byref(nbytes),
                                                   C.byref(chunks)))
        return {"device_ms": ms.value, "rows": rows.value, "bytes": nbytes.value, "chunks": chunks.value}

    _close_order = 1

    def close(self) -> None:
        if getattr(self, "h", None):
            if self.ctx.h:
                self.ctx.lib.qm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchResults:
    """The n results of a batch run; each Result is wrapped on first access
    (unaccessed handles are destroyed with this object)."""

    def __init__(self, lib, handles: list[int]):
        self.lib = lib
        self.handles = handles
        self.cache: dict[int, Result] = {}

    def __len__(self) -> int:
        return len(self.handles)

    def __getitem__(self, i: int) -> Result:
        if i not in self.cache:
            self.cache[i] = Result.from_handle(self.lib, C.c_void_p(self.handles[i]), owned=True)
        return self.cache[i]

    def __iter__(self):
        for i in range(len(self.handles)):
            yield self[i]

    def __del__(self):
        try:
            for i, h in enumerate(self.handles):
                if i not in self.cache and h:
                    self.lib.qm_result_destroy(C.c_void_p(h))
        except Exception:
            pass


class Server:
    """A qm_server: native lanes (worker threads, each with its own CUDA
    stream) that take submitted requests over resident tables as batched
    launches while other lanes' batches run, within an HBM budget.  Requests
    over tables of more than max_batch_rows rows, or planned at more than
    max_batch_groups groups, run alone; the last lane takes small requests
    only.  While it runs, the context is the server's:
    register tables first."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int, max_batch: int = 64, max_wait_us: int = 0,
                 max_batch_rows: int = 0, lanes: int = 0, max_batch_groups: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = A.QmServerConfig(hbm_budget_bytes, max_batch, max_wait_us, max_batch_rows, lanes, max_batch_groups)
        h = C.c_void_p()
        ctx.check(self.lib.qm_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        ctx._adopt(self)
        self._queries: dict[int, CQuery] = {}

    def submit(self, table: Table, query) -> int:
        cq = query if isinstance(query, CQuery) else CQuery(query)
        t = C.c_uint64()
        status = self.lib.qm_server_submit(self.h, table.h, C.byref(cq.struct), C.byref(t))
        if status != A.QM_OK:
            raise A.QmError(status, "submit")
        return t.value

    def cancel(self, ticket: int) -> bool:
        return self.lib.qm_server_cancel(self.h, ticket) == A.QM_OK

    def wait(self, ticket: int, timeout_s: float | None = None) -> tuple["Result", dict]:
        """The request's Result and timing (µs); raises QmError with the
        request's own status and message if it failed or was cancelled."""
        out = C.c_void_p()
        tm = A.QmServerTiming()
        msg = C.create_string_buffer(512)
        tmo = -1 if timeout_s is None else int(timeout_s * 1e6)
        status = self.lib.qm_server_wait(self.h, ticket, tmo, C.byref(out), C.byref(tm), msg, len(msg))
        timing = {"queued_us": tm.queued_us, "run_us": tm.run_us, "total_us": tm.total_us,
                  "batch_size": tm.batch_size, "plan_us": tm.plan_us}
        if status != A.QM_OK:
            raise A.QmError(status, msg.value.decode(errors="replace"))
        return Result.from_handle(self.lib, out, owned=True), timing

    def stats(self) -> dict:
        c = A.QmServerCounters()
        _check(self.lib, None, self.lib.qm_server_stats(self.h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in A.QmServerCounters._fields_}

    _close_order = 0

    def close(self) -> None:
        if getattr(self, "h", None):
            if self.ctx.h:
                self.lib.qm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
