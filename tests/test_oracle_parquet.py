"""The oracle's restatement of the reference's PLAIN column-chunk decode,
pinned to the reference's own fixture (tests/golden/parquet_plain.json) and
to pyarrow on written files (v1 and v2 pages, NULLs, several pages)."""
import base64
import json
import math
import os
import struct

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


DICT_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "parquet_dict.json")


def load_dict_fixture():
    import hashlib
    import zlib
    g = json.load(open(DICT_GOLDEN))
    chunk = zlib.decompress(open(os.path.join(os.path.dirname(DICT_GOLDEN), g["chunk_file"]), "rb").read())
    assert hashlib.sha256(chunk).hexdigest() == g["chunk_sha256"]
    return g, chunk


def test_reference_dictionary_fixture():
    # benchmark_100k_uncompressed.parquet's id: a 100,000-value dictionary
    # page and one v1 page of 17-bit RLE_DICTIONARY indices
    g, chunk = load_dict_fixture()
    assert decode_column_chunk(chunk, PHYS[g["physical_type"]], g["num_values"]) == list(range(g["num_values"]))


@pytest.mark.parametrize("version", ["1.0", "2.0"])
@pytest.mark.parametrize("dict_limit", [1 << 20, 2048])
def test_dictionary_files_match_pyarrow(version, dict_limit):
    # dict_limit 2048: the dictionary outgrows it and later pages are PLAIN.
    # v1 pages of a dictionary still growing while they were written carry a
    # narrower index bit width than the final dictionary's, so the
    # reference's level-section test (the byte after the levels must equal
    # ceil(log2(dictionary size))) misses their levels and it decodes them
    # differently from pyarrow (the i64 / f64 columns below); the oracle
    # follows the reference there, and is held to pyarrow everywhere else.
    import io

    import pyarrow.parquet as pq

    from tests.parquet_util import dict_columns, write_dict
    raw = write_dict(dict_columns(20000, 4), version, page_size=1024, dict_limit=dict_limit)
    table = pq.read_table(io.BytesIO(raw))
    growing = version == "1.0" and dict_limit > 4096
    for name, phys, chunk, nv in chunks_of(raw):
        vals = decode_column_chunk(chunk, PHYS[phys], nv)
        want = table.column(name).to_pylist()
        assert len(vals) == len(want)
        same = all(_same(a, b) for a, b in zip(vals, want))
        assert same != (growing and name in ("i64", "f64")), name


def test_corrupt_chunks_terminate():
    # byte flips and truncations: the restatement ends (decoding, or raising
    # where it would read past the bytes) and never spins on a corrupt count
    import time

    import numpy as np

    from tests.parquet_util import dict_columns, write_dict
    rng = np.random.default_rng(32)
    raws = [write_plain(sample_columns(2000, 2), "1.0", page_size=512),
            write_dict(dict_columns(2000, 4), "1.0", page_size=512),
            write_dict(dict_columns(2000, 5), "2.0", page_size=512)]
    t0 = time.time()
    for raw in raws:
        for nm, ph, ch, nv in chunks_of(raw):
            for trial in range(40):
                b = bytearray(ch)
                for _ in range(int(rng.integers(1, 8))):
                    b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
                if trial % 4 == 0:
                    b = b[:int(rng.integers(1, len(b)))]
                try:
                    vals = decode_column_chunk(bytes(b), PHYS[ph], nv)
                    assert len(vals) <= nv
                except (IndexError, ValueError, NotImplementedError, struct.error):
                    pass
    assert time.time() - t0 < 60
