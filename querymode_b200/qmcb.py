"""QMCB columnar batch codec for numeric columns.

Layout (src/columnar.ts:438-613, docs/src/content/docs/columnar-format.mdx:25-44):
header magic u32 0x42434D51, rowCount u32, colCount u16; per column
nameLen u16, name (UTF-8), dtype u8, hasNulls u8; then per column an optional
null bitmap (ceil(rows/8) bytes, bit set = NULL, LSB first) followed by the
packed little-endian values.  Only the numeric dtypes the GPU path reads are
produced or decoded (F64=0, I64=1, I32=6, F32=7).
"""
from __future__ import annotations

import struct
from typing import Any, Mapping

import numpy as np

from . import _abi as A
from .engine import Column, ResultColumn, pack_nulls, unpack_nulls

QMCB_MAGIC = 0x42434D51
_DT = {A.QM_F64: np.float64, A.QM_I64: np.int64, A.QM_I32: np.int32, A.QM_F32: np.float32}
_TAG = {np.dtype(np.float64): A.QM_F64, np.dtype(np.int64): A.QM_I64,
        np.dtype(np.int32): A.QM_I32, np.dtype(np.float32): A.QM_F32}


def encode(columns: Mapping[str, Any]) -> bytes:
    """encodeColumnarBatch for numeric columns (arrays or engine.Column)."""
    items = []
    n = None
    for name, v in columns.items():
        nulls = None
        if isinstance(v, Column):
            v, nulls = v.values, v.nulls
        arr = np.ascontiguousarray(v)
        if arr.dtype not in _TAG:
            raise TypeError(f"{name}: {arr.dtype} is not a QMCB numeric dtype")
        if n is None:
            n = arr.size
        elif arr.size != n:
            raise ValueError("columns differ in length")
        items.append((name, arr, pack_nulls(nulls)))
    n = n or 0
    out = [struct.pack("<IIH", QMCB_MAGIC, n, len(items))]
    for name, arr, nb in items:
        nm = name.encode()
        out.append(struct.pack("<H", len(nm)) + nm + struct.pack("<BB", _TAG[arr.dtype], 1 if nb is not None else 0))
    for name, arr, nb in items:
        if nb is not None:
            out.append(nb.tobytes()[: (n + 7) // 8].ljust((n + 7) // 8, b"\0"))
        out.append(arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes())
    return b"".join(out)


class Decoded:
    def __init__(self, columns: list[ResultColumn], n_rows: int):
        self.columns = columns
        self.n_rows = n_rows

    @property
    def names(self) -> list[str]:
        return [c.name for c in self.columns]

    def column(self, name: str) -> ResultColumn:
        for c in self.columns:
            if c.name == name:
                return c
        raise KeyError(name)


def decode(buf: bytes) -> Decoded:
    """decodeColumnarBatch for numeric columns (other dtypes are skipped)."""
    if len(buf) < 10:
        raise ValueError("QMCB buffer shorter than its header")
    magic, n, nc = struct.unpack_from("<IIH", buf, 0)
    if magic != QMCB_MAGIC:
        raise ValueError("bad QMCB magic")
    pos = 10
    descs = []
    for _ in range(nc):
        (ln,) = struct.unpack_from("<H", buf, pos)
        pos += 2
        name = buf[pos:pos + ln].decode()
        pos += ln
        dt, hn = struct.unpack_from("<BB", buf, pos)
        pos += 2
        descs.append((name, dt, hn))
    cols = []
    for name, dt, hn in descs:
        nulls = None
        if hn:
            nb = (n + 7) // 8
            nulls = unpack_nulls(np.frombuffer(buf, np.uint8, nb, pos), n)
            pos += nb
        if dt not in _DT:
            raise ValueError(f"{name}: QMCB dtype {dt} is not numeric")
        size = np.dtype(_DT[dt]).itemsize * n
        vals = np.frombuffer(buf[pos:pos + size], dtype=np.dtype(_DT[dt]).newbyteorder("<")).astype(_DT[dt])
        pos += size
        cols.append(ResultColumn(name, dt, False, vals, nulls))
    return Decoded(cols, n)
