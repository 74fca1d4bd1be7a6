"""Parquet files for the decode tests, written with pyarrow: PLAIN pages,
uncompressed, data page v1 or v2, small pages (several per chunk)."""
import io

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq

PHYS = {"INT32": "int32", "INT64": "int64", "FLOAT": "float32", "DOUBLE": "float64"}


def write_plain(cols: dict, version: str, page_size: int = 4096) -> bytes:
    arrays = {}
    for name, (vals, mask) in cols.items():
        arrays[name] = pa.array(vals, mask=mask)
    buf = io.BytesIO()
    pq.write_table(pa.table(arrays), buf, use_dictionary=False, compression="NONE",
                   data_page_version=version, data_page_size=page_size, write_statistics=True)
    return buf.getvalue()


def write_dict(cols: dict, version: str, page_size: int = 4096, dict_limit: int = 1 << 20) -> bytes:
    """Dictionary-encoded (RLE_DICTIONARY indices; PLAIN pages after the
    dictionary outgrows `dict_limit` bytes), uncompressed."""
    arrays = {name: pa.array(vals, mask=mask) for name, (vals, mask) in cols.items()}
    buf = io.BytesIO()
    pq.write_table(pa.table(arrays), buf, use_dictionary=True, compression="NONE", data_page_version=version,
                   data_page_size=page_size, dictionary_pagesize_limit=dict_limit, write_statistics=True)
    return buf.getvalue()


def dict_columns(n: int, seed: int):
    """Few distinct values per column (dictionary-friendly), NULLs in some."""
    rng = np.random.default_rng(seed)
    return {
        "i32": (rng.integers(-50, 50, n).astype(np.int32), rng.random(n) < 0.1),
        "i64": ((rng.integers(0, 3000, n) * 7919 - 10**12).astype(np.int64), None),
        "f32": (rng.integers(0, 7, n).astype(np.float32) / 4, rng.random(n) < 0.3),
        "f64": (rng.integers(0, 20000, n) * 0.5, None),
        "key": (((np.arange(n) * 7919) % 101).astype(np.int64), None),
    }


def chunks_of(raw: bytes):
    """(name, physical type, chunk bytes, num_values) of row group 0."""
    md = pq.ParquetFile(io.BytesIO(raw)).metadata.row_group(0)
    out = []
    for c in range(md.num_columns):
        cc = md.column(c)
        start = cc.dictionary_page_offset if cc.dictionary_page_offset is not None else cc.data_page_offset
        out.append((cc.path_in_schema, cc.physical_type, raw[start:start + cc.total_compressed_size], cc.num_values))
    return out


def sample_columns(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return {
        "i32": (rng.integers(-2**31, 2**31 - 1, n).astype(np.int32), rng.random(n) < 0.1),
        "i64": (rng.integers(-2**62, 2**62, n).astype(np.int64), rng.random(n) < 0.3),
        "f32": (rng.normal(size=n).astype(np.float32), None),
        "f64": (rng.normal(size=n) * 1e3, np.arange(n) % 7 == 0),
        "key": (((np.arange(n) * 7919) % 101).astype(np.int64), None),
    }
