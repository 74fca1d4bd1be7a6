"""The oracle's restatement of the reference's PLAIN column-chunk decode,
pinned to the reference's own fixture (tests/golden/parquet_plain.json) and
to pyarrow on written files (v1 and v2 pages, NULLs, several pages)."""
import base64
import json
import math
import os

import pytest

from oracle.parquet import decode_column_chunk
from tests.parquet_util import PHYS, chunks_of, sample_columns, write_plain

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "parquet_plain.json")


def _same(a, b):
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, float) and math.isnan(a):
        return isinstance(b, float) and math.isnan(b)
    return a == b


def test_reference_fixture():
    g = json.load(open(GOLDEN))
    assert {c["name"] for c in g["columns"]} == {"id", "value"}
    for c in g["columns"]:
        vals = decode_column_chunk(base64.b64decode(c["chunk"]), PHYS[c["physical_type"]], c["num_values"])
        assert vals == c["values"]


@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_written_files_match_pyarrow(version):
    import io

    import pyarrow.parquet as pq
    raw = write_plain(sample_columns(5000, 3), version, page_size=2048)
    table = pq.read_table(io.BytesIO(raw))
    for name, phys, chunk, nv in chunks_of(raw):
        vals = decode_column_chunk(chunk, PHYS[phys], nv)
        want = table.column(name).to_pylist()
        assert len(vals) == len(want)
        assert all(_same(a, b) for a, b in zip(vals, want)), name
