"""Parquet PLAIN column chunks decoded on the device (qm_table_from_parquet)
against the reference's decode restated (oracle/parquet.py): the same rows,
values and NULLs; then a query over the decoded table against the oracle."""
import base64
import io
import json
import os

import numpy as np
import pytest

import oracle
from oracle.parquet import decode_column_chunk
from querymode_b200 import _abi as A
from querymode_b200.engine import Column
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same
from tests.parquet_util import PHYS, chunks_of, sample_columns, write_plain

pytestmark = pytest.mark.gpu

QM = {"INT32": A.QM_I32, "INT64": A.QM_I64, "FLOAT": A.QM_F32, "DOUBLE": A.QM_F64}
NP = {"INT32": np.int32, "INT64": np.int64, "FLOAT": np.float32, "DOUBLE": np.float64}


def check_decoded(t, name, phys, chunk, nv):
    vals, nulls = t.read_column(name)
    want = decode_column_chunk(chunk, PHYS[phys], nv)
    assert len(vals) == len(want)
    wn = np.array([w is None for w in want])
    assert np.array_equal(nulls, wn), name
    wv = np.array([0 if w is None else w for w in want], dtype=NP[phys])
    if phys in ("FLOAT", "DOUBLE"):  # NaN payloads are not observable in the reference's numbers
        nan = np.isnan(wv)
        assert np.array_equal(np.isnan(vals), nan), name
        vals, wv = vals[~nan], wv[~nan]
    assert np.array_equal(vals.view(np.uint8), wv.view(np.uint8)), name  # bit-exact, zeros where NULL


def test_reference_fixture(ctx):
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "parquet_plain.json")))
    chunks = [(c["name"], QM[c["physical_type"]], base64.b64decode(c["chunk"]), c["num_values"]) for c in g["columns"]]
    t = ctx.table_from_parquet_chunks(chunks)
    for c in g["columns"]:
        vals, nulls = t.read_column(c["name"])
        assert vals.tolist() == c["values"] and not nulls.any()


@pytest.mark.parametrize("version", ["1.0", "2.0"])
@pytest.mark.parametrize("n,page", [(50_000, 4096), (1_000_003, 1 << 20), (7, 64)])
def test_written_files(ctx, tmp_path, version, n, page):
    raw = write_plain(sample_columns(n, 5), version, page_size=page)
    chunks = chunks_of(raw)
    t = ctx.table_from_parquet_chunks([(nm, QM[ph], ch, nv) for nm, ph, ch, nv in chunks])
    assert t.n_rows == n
    for nm, ph, ch, nv in chunks:
        check_decoded(t, nm, ph, ch, nv)
    # and a query over the decoded table, against the oracle over the same data
    path = tmp_path / "t.parquet"
    path.write_bytes(raw)
    t2 = ctx.table_from_parquet(str(path))
    cols = {}
    for nm, ph, ch, nv in chunks:
        vals, nulls = t2.read_column(nm)
        cols[nm] = Column(vals, nulls if nulls.any() else None)
    q = QueryDescriptor(filters=[FilterOp("i32", "gt", 0)], group_by=["key"],
                        aggregates=[AggregateOp("sum", "f64"), AggregateOp("count", "i64"), AggregateOp("max", "f32"),
                                    AggregateOp("sum", "i64")])
    assert_same(t2.run(q), oracle.run(cols, q))


def test_reference_dictionary_fixture(ctx):
    # benchmark_100k_uncompressed.parquet's id chunk: 100,000-entry dictionary,
    # 17-bit bit-packed indices
    from tests.test_oracle_parquet import load_dict_fixture
    g, chunk = load_dict_fixture()
    t = ctx.table_from_parquet_chunks([(g["column"], QM[g["physical_type"]], chunk, g["num_values"])])
    vals, nulls = t.read_column(g["column"])
    assert not nulls.any() and np.array_equal(vals, np.arange(g["num_values"], dtype=np.int64))


@pytest.mark.parametrize("version", ["1.0", "2.0"])
@pytest.mark.parametrize("dict_limit", [1 << 20, 2048])
def test_dictionary_files(ctx, tmp_path, version, dict_limit):
    # RLE_DICTIONARY pages (and PLAIN ones once the dictionary outgrows its
    # limit) against the oracle, including the v1 pages the reference reads
    # without their levels; then a query over the decoded table
    from tests.parquet_util import dict_columns, write_dict
    raw = write_dict(dict_columns(60_000, 6), version, page_size=2048, dict_limit=dict_limit)
    chunks = chunks_of(raw)
    t = ctx.table_from_parquet_chunks([(nm, QM[ph], ch, nv) for nm, ph, ch, nv in chunks])
    cols = {}
    for nm, ph, ch, nv in chunks:
        check_decoded(t, nm, ph, ch, nv)
        vals, nulls = t.read_column(nm)
        cols[nm] = Column(vals, nulls if nulls.any() else None)
    q = QueryDescriptor(filters=[FilterOp("i32", "gt", -20)], group_by=["key"],
                        aggregates=[AggregateOp("sum", "f64"), AggregateOp("count", "*"), AggregateOp("max", "f32"),
                                    AggregateOp("sum", "i64"), AggregateOp("min", "i64")])
    assert_same(t.run(q), oracle.run(cols, q))


def test_unsupported_pages(ctx, tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    tab = pa.table({"x": pa.array(np.arange(1000, dtype=np.int64) % 10)})
    # PLAIN_DICTIONARY data pages (file format 1.0; the reference would read
    # them as PLAIN) and compressed pages
    for kw in ({"use_dictionary": True, "compression": "NONE", "version": "1.0"},
               {"use_dictionary": False, "compression": "SNAPPY"}):
        p = tmp_path / "u.parquet"
        pq.write_table(tab, p, **kw)
        with pytest.raises(A.QmError) as e:
            ctx.table_from_parquet(str(p))
        assert e.value.status == A.QM_ERR_UNSUPPORTED


def test_corrupt_chunks_are_refused_or_decoded(ctx):
    # byte flips and truncations of real chunks: the host parser must stay
    # inside the bytes given and end; each call builds a table or returns an
    # error code, and a table it builds decodes as the oracle does
    from tests.parquet_util import dict_columns, write_dict
    rng = np.random.default_rng(31)
    raws = [write_plain(sample_columns(3000, 2), "1.0", page_size=512),
            write_plain(sample_columns(3000, 3), "2.0", page_size=512),
            write_dict(dict_columns(3000, 4), "1.0", page_size=512),
            write_dict(dict_columns(3000, 5), "2.0", page_size=512)]
    built = 0
    for raw in raws:
        for nm, ph, ch, nv in chunks_of(raw):
            for trial in range(30):
                b = bytearray(ch)
                for _ in range(int(rng.integers(1, 6))):
                    b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
                if trial % 3 == 0:
                    b = b[:int(rng.integers(1, len(b)))]
                try:
                    t = ctx.table_from_parquet_chunks([(nm, QM[ph], bytes(b), nv)])
                except A.QmError:
                    continue
                built += 1
                try:
                    decode_column_chunk(bytes(b), PHYS[ph], nv)
                except Exception:  # the restatement reads past the bytes: no reference answer
                    t.close()
                    continue
                check_decoded(t, nm, ph, bytes(b), nv)
                t.close()
    assert built > 0
