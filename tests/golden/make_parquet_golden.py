"""Writes tests/golden/parquet_plain.json from the reference's own Parquet
test fixture wasm/tests/fixtures/simple_plain.parquet (PLAIN pages, optional
INT64 and DOUBLE columns): each numeric column chunk's bytes (from its first
page header) with ColumnMetaData.num_values and the values the reference's
test expects (tests/test_parquet.zig reads this file; pyarrow decodes it
here as the expected values).  Also tests/golden/parquet_dict_id.bin.zlib +
parquet_dict.json from wasm/tests/fixtures/benchmark_100k_uncompressed.parquet:
its `id` column chunk (a dictionary page of 100,000 INT64 values and one v1
data page of 17-bit RLE_DICTIONARY indices), zlib-compressed, whose values
pyarrow decodes as 0..99,999.  Run where the reference is checked out:

    python tests/golden/make_parquet_golden.py <path to the reference checkout>
"""
import base64
import hashlib
import json
import os
import sys
import zlib

import pyarrow.parquet as pq


def main(ref_root: str) -> None:
    path = os.path.join(ref_root, "wasm", "tests", "fixtures", "simple_plain.parquet")
    raw = open(path, "rb").read()
    md = pq.ParquetFile(path).metadata.row_group(0)
    table = pq.read_table(path)
    cols = []
    for c in range(md.num_columns):
        cc = md.column(c)
        if cc.physical_type not in ("INT32", "INT64", "FLOAT", "DOUBLE"):
            continue
        start = cc.dictionary_page_offset if cc.dictionary_page_offset is not None else cc.data_page_offset
        cols.append({"name": cc.path_in_schema, "physical_type": cc.physical_type,
                     "num_values": cc.num_values,
                     "chunk": base64.b64encode(raw[start:start + cc.total_compressed_size]).decode(),
                     "values": table.column(cc.path_in_schema).to_pylist()})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "parquet_plain.json")
    with open(out, "w") as f:
        json.dump({"source": "wasm/tests/fixtures/simple_plain.parquet", "columns": cols}, f, indent=1)

    # the dictionary-encoded fixture's id column
    path = os.path.join(ref_root, "wasm", "tests", "fixtures", "benchmark_100k_uncompressed.parquet")
    raw = open(path, "rb").read()
    md = pq.ParquetFile(path).metadata.row_group(0)
    cc = next(md.column(c) for c in range(md.num_columns) if md.column(c).path_in_schema == "id")
    start = cc.dictionary_page_offset
    chunk = raw[start:start + cc.total_compressed_size]
    values = pq.read_table(path).column("id").to_pylist()
    assert values == list(range(cc.num_values))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "parquet_dict_id.bin.zlib"), "wb") as f:
        f.write(zlib.compress(chunk, 9))
    with open(os.path.join(here, "parquet_dict.json"), "w") as f:
        json.dump({"source": "wasm/tests/fixtures/benchmark_100k_uncompressed.parquet", "column": "id",
                   "physical_type": cc.physical_type, "num_values": cc.num_values,
                   "chunk_file": "parquet_dict_id.bin.zlib", "chunk_sha256": hashlib.sha256(chunk).hexdigest(),
                   "values": "0 .. num_values - 1"}, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_parquet_golden.py <path to the reference checkout>")
    main(sys.argv[1])
