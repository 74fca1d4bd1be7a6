"""Test infrastructure: the reference's scan-page decode restated, to check
the device decoder against.

Follows src/decode.ts: decodePage (:251-331) for numeric dtypes — an
optional validity bitmap (ceil(rowCount/8) bytes, bit set = a value) when
nullCount > 0 and rowCount > 0, then either the non-NULL values packed
(Parquet-style) or, from dataOffsetInPage, one slot per row (Lance v2
nullable pages); decodePlainValues (src/parquet-decode.ts:280-386) caps the
values at what the bytes hold — and decodeAllColumns (:201-229), which
decodes a column's pages in order and concatenates them, a page with an
encoding going through decodeParquetColumnChunk.  Values come back as Python
numbers with None for NULL.
"""
from __future__ import annotations

from .parquet import decode_column_chunk, decode_plain

MAX_SAFE_INTEGER = 2**53 - 1


def decode_page(buf: bytes, dtype: str, null_count: int = 0, row_count: int = 0,
                data_offset: int | None = None) -> list:
    """decodePage (src/decode.ts:251-331) for int32 / int64 / float32 / float64."""
    bitmap = None
    if null_count > 0 and row_count > 0:
        nbytes = (row_count + 7) // 8
        if len(buf) < nbytes:
            return []
        bitmap = buf[:nbytes]
        strip = nbytes if data_offset is None else data_offset
        buf = buf[strip:]
    slotted = data_offset is not None
    if row_count > 0:
        n = row_count if slotted else row_count - (null_count if bitmap is not None else 0)
    else:
        n = MAX_SAFE_INTEGER
    values = decode_plain(buf, dtype, max(n, 0))
    if bitmap is None:
        return values

    def is_null(i):
        return not (bitmap[i >> 3] >> (i & 7)) & 1

    if slotted:
        return [None if is_null(i) else v for i, v in enumerate(values)]
    out, vi = [], 0
    for i in range(row_count):
        if is_null(i):
            out.append(None)
        elif vi < len(values):
            out.append(values[vi])
            vi += 1
        else:
            out.append(None)
    return out


def decode_column_pages(pages: list, dtype: str) -> list:
    """decodeAllColumns (src/decode.ts:201-229) for one column: `pages` are
    (buf, row_count, null_count, data_offset, parquet) tuples."""
    out = []
    for buf, row_count, null_count, data_offset, parquet in pages:
        if parquet:
            out += decode_column_chunk(buf, dtype, row_count)
        else:
            out += decode_page(buf, dtype, null_count, row_count, data_offset)
    return out
