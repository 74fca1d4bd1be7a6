"""Scan pages decoded on the device (qm_table_from_pages) against the
reference's decodePage / decodeAllColumns restated (oracle/pages.py): the
reference's known answers, seeded pages of every layout including short and
inconsistent ones, Parquet chunks among them, then a query over a table
built from pages against the oracle."""
import struct

import numpy as np
import pytest

import oracle
from oracle.pages import decode_column_pages
from querymode_b200 import _abi as A
from querymode_b200.engine import Column, Page, PageTable
from querymode_b200.query import AggregateOp, FilterOp, QueryDescriptor
from tests.helpers import assert_same
from tests.page_util import as_tuples, encode_column, encode_page
from tests.parquet_util import chunks_of, write_plain

pytestmark = pytest.mark.gpu

QM = {"int32": A.QM_I32, "int64": A.QM_I64, "float32": A.QM_F32, "float64": A.QM_F64}
NP = {"int32": np.int32, "int64": np.int64, "float32": np.float32, "float64": np.float64}


def check_column(t, name, dtype, pages):
    vals, nulls = t.read_column(name)
    want = decode_column_pages(as_tuples(pages), dtype)
    assert len(vals) == len(want), name
    wn = np.array([w is None for w in want], dtype=bool)
    assert np.array_equal(nulls, wn), name
    wv = np.array([0 if w is None else w for w in want], dtype=NP[dtype])
    if dtype.startswith("float"):  # NaN payloads are not observable in the reference's numbers
        nan = np.isnan(wv)
        assert np.array_equal(np.isnan(vals), nan), name
        vals, wv = vals[~nan], wv[~nan]
    assert np.array_equal(vals.view(np.uint8), wv.view(np.uint8)), name  # bit-exact (+0 / -0 included)


def test_reference_known_answers(ctx):  # src/decode.test.ts:11-99
    cases = [("int32", [Page(struct.pack("<3i", 100, -50, 0))], [100, -50, 0]),
             ("int64", [Page(struct.pack("<2q", 9007199254740993, -42))], [9007199254740993, -42]),
             ("int32", [Page(bytes([0x05]) + struct.pack("<2i", 100, 300), 3, 1)], [100, None, 300])]
    for dtype, pages, want in cases:
        t = ctx.table_from_pages([("c", QM[dtype], pages)])
        vals, nulls = t.read_column("c")
        assert [None if z else v for v, z in zip(vals.tolist(), nulls.tolist())] == want
    t = ctx.table_from_pages([("c", A.QM_F32, [Page(struct.pack("<2f", 3.14, -2.718))])])
    vals, _ = t.read_column("c")
    assert vals.tolist() == pytest.approx([3.14, -2.718], abs=5e-3)


def random_pages(rng, dtype, n_pages):
    w = np.dtype(NP[dtype]).itemsize
    pages = []
    for _ in range(n_pages):
        n = int(rng.integers(0, 3000))
        if dtype.startswith("int"):
            vals = rng.integers(np.iinfo(NP[dtype]).min, np.iinfo(NP[dtype]).max, n, dtype=NP[dtype])
        else:
            vals = (rng.normal(size=n) * 1e6).astype(NP[dtype])
        mask = rng.random(n) < rng.choice([0.0, 0.05, 0.5, 1.0])
        kind = rng.integers(0, 9)
        if kind == 7:  # a Parquet chunk among the pages
            raw = write_plain({"c": (vals, mask if mask.any() else None)}, rng.choice(["1.0", "2.0"]),
                              page_size=int(rng.choice([512, 4096])))
            _, _, chunk, nv = chunks_of(raw)[0]
            pages.append(Page(chunk, nv, 0, None, True))
            continue
        p = encode_page(vals, mask, ["plain", "packed", "slotted"][kind % 3], pad=int(rng.choice([1, 8, 64])))
        buf = p.buf
        if kind == 3:    # cut short at a random byte
            buf = buf[:int(rng.integers(0, len(buf) + 1))]
        elif kind == 4:  # rowCount 0: every value the bytes hold
            p = Page(buf, 0, p.null_count, p.data_offset)
        elif kind == 5:  # nullCount that disagrees with the bitmap
            p = Page(buf, p.row_count, int(rng.integers(1, max(2, p.row_count + 3))), p.data_offset)
        elif kind == 6 and p.data_offset is not None:  # slot offset past the end
            p = Page(buf, p.row_count, p.null_count, len(buf) + int(rng.integers(0, 16)))
        pages.append(Page(buf, p.row_count, p.null_count, p.data_offset))
    return pages


@pytest.mark.parametrize("dtype", ["int32", "int64", "float32", "float64"])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_pages(ctx, dtype, seed):
    rng = np.random.default_rng(seed * 10 + len(dtype))
    pages = random_pages(rng, dtype, 40)
    t = ctx.table_from_pages([("c", QM[dtype], pages)])
    check_column(t, "c", dtype, pages)


def test_unaligned_values(ctx):
    # packed values behind a 1-byte bitmap (odd offsets) and Parquet PLAIN values at any offset
    rng = np.random.default_rng(7)
    vals = rng.integers(-2**62, 2**62, 1001, dtype=np.int64)
    mask = rng.random(1001) < 0.3
    pages = [encode_page(vals[a:a + 7], mask[a:a + 7], "packed") for a in range(0, 1001, 7)]
    t = ctx.table_from_pages([("c", A.QM_I64, pages)])
    check_column(t, "c", "int64", pages)


def test_query_over_pages(ctx):
    rng = np.random.default_rng(11)
    n = 300_000
    key = (rng.zipf(1.3, n) % 1000).astype(np.int64)
    qty = rng.integers(1, 100, n).astype(np.int32)
    price = rng.random(n) * 1000
    pmask = rng.random(n) < 0.05
    qmask = rng.random(n) < 0.02
    cols = [("key", A.QM_I64, encode_column(key, None, 10_000)),
            ("qty", A.QM_I32, encode_column(qty, qmask, 10_000, ("packed", "slotted"), rng)),
            ("price", A.QM_F64, encode_column(price, pmask, 10_000, ("packed", "slotted", "plain"), rng))]
    t = ctx.table_from_pages(cols)
    assert t.n_rows == n
    ref_cols = {}
    for name, qd, pages in cols:  # the oracle's decode of the same pages ("plain" pages drop the NULLs)
        dt = {A.QM_I64: "int64", A.QM_I32: "int32", A.QM_F64: "float64"}[qd]
        dec = decode_column_pages(as_tuples(pages), dt)
        nulls = np.array([v is None for v in dec])
        ref_cols[name] = Column(np.array([0 if v is None else v for v in dec], dtype=NP[dt]), nulls if nulls.any() else None)
    assert ref_cols["price"].nulls.sum() < pmask.sum()
    q = QueryDescriptor(filters=[FilterOp("qty", "gt", 10)], group_by=["key"],
                        aggregates=[AggregateOp("sum", "price"), AggregateOp("sum", "qty"), AggregateOp("min", "price"),
                                    AggregateOp("max", "price"), AggregateOp("count", "*"), AggregateOp("avg", "price")])
    assert_same(t.run(q), oracle.run(ref_cols, q))


def test_bad_descriptors(ctx):
    with pytest.raises(A.QmError) as e:
        ctx.table_from_pages([("a", A.QM_I32, [Page(bytes(8))]), ("b", A.QM_I32, [Page(bytes(12))])])
    assert e.value.status == A.QM_ERR_INVALID
    with pytest.raises(A.QmError) as e:
        ctx.table_from_pages([("a", A.QM_I32, [Page(bytes(8), 2, 0, -5)])])
    assert e.value.status == A.QM_ERR_INVALID


def test_page_table_matches_page_list(ctx):
    """A column's pages back to back in one buffer with a page table decode
    as the same pages passed one by one."""
    rng = np.random.default_rng(21)
    pages = random_pages(rng, "int64", 30)
    pages = [p for p in pages if not p.parquet]
    bufs = [bytes(p.buf) for p in pages]
    lens = np.array([len(b) for b in bufs], dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    pt = PageTable(np.frombuffer(b"".join(bufs), dtype=np.uint8), offs, lens,
                   np.array([p.row_count for p in pages]), np.array([p.null_count for p in pages]),
                   np.array([-1 if p.data_offset is None else p.data_offset for p in pages]))
    t1 = ctx.table_from_pages([("c", A.QM_I64, pages)])
    t2 = ctx.table_from_pages([("c", A.QM_I64, pt)])
    v1, n1 = t1.read_column("c")
    v2, n2 = t2.read_column("c")
    assert np.array_equal(v1, v2) and np.array_equal(n1, n2)
    check_column(t2, "c", "int64", pages)


def test_pinned_page_buffers(ctx):
    """Pages in page-locked memory go to the device without staging; back to
    back in one buffer they are one copy, at the buffer's own alignment."""
    import torch
    rng = np.random.default_rng(23)
    for dtype in ("int32", "int64", "float64"):
        pages = [p for p in random_pages(rng, dtype, 25) if not p.parquet]
        bufs = [bytes(p.buf) for p in pages]
        lens = np.array([len(b) for b in bufs], dtype=np.int64)
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
        joined = np.frombuffer(b"".join(bufs), dtype=np.uint8)
        pinned = torch.from_numpy(joined.copy()).pin_memory().numpy()
        args = (offs, lens, np.array([p.row_count for p in pages]), np.array([p.null_count for p in pages]),
                np.array([-1 if p.data_offset is None else p.data_offset for p in pages]))
        t1 = ctx.table_from_pages([("c", QM[dtype], PageTable(joined, *args))])
        t2 = ctx.table_from_pages([("c", QM[dtype], PageTable(pinned, *args))])
        v1, n1 = t1.read_column("c")
        v2, n2 = t2.read_column("c")
        assert np.array_equal(v1.view(np.uint8), v2.view(np.uint8)) and np.array_equal(n1, n2), dtype
        check_column(t2, "c", dtype, pages)
        t1.close()
        t2.close()


def test_empty_inputs(ctx):
    """Empty pages, an empty page table and a Parquet chunk of no values make
    a table of 0 rows; the ungrouped aggregate over it answers as the oracle."""
    from tests.parquet_util import chunks_of, write_plain
    raw = write_plain({"c": (np.zeros(0, dtype=np.int64), None)}, "1.0")
    _, _, chunk, nv = chunks_of(raw)[0]
    empty_pt = PageTable(np.zeros(0, dtype=np.uint8), np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64))
    specs = [[("c", A.QM_I64, [Page(b""), Page(b"", 0, 0), Page(bytes([0xFF]), 9, 1)])],
             [("c", A.QM_I64, empty_pt)],
             [("c", A.QM_I64, [Page(chunk, nv, 0, None, True)])],
             [("c", A.QM_I64, [])]]
    q = QueryDescriptor(aggregates=[AggregateOp("sum", "c"), AggregateOp("count", "*"), AggregateOp("max", "c")])
    for spec in specs:
        t = ctx.table_from_pages(spec)
        assert t.n_rows == 0
        vals, nulls = t.read_column("c")
        assert len(vals) == 0 and len(nulls) == 0
        assert_same(t.run(q), oracle.run({"c": np.zeros(0, dtype=np.int64)}, q))
        t.close()


NARROW = {"int8": (A.QM_PT_INT8, A.QM_I32, np.int8, np.int32), "uint8": (A.QM_PT_UINT8, A.QM_I32, np.uint8, np.int32),
          "int16": (A.QM_PT_INT16, A.QM_I32, np.int16, np.int32), "uint16": (A.QM_PT_UINT16, A.QM_I32, np.uint16, np.int32),
          "uint32": (A.QM_PT_UINT32, A.QM_F64, np.uint32, np.float64),
          "float16": (A.QM_PT_FLOAT16, A.QM_F32, np.float16, np.float32)}


@pytest.mark.parametrize("src", list(NARROW))
def test_narrow_page_types(ctx, src):
    """Pages of int8 / uint8 / int16 / uint16 / uint32 / float16 values are
    widened on the device to the cells the reference's numbers hold (int32,
    double, float), bit for bit against the oracle's decode."""
    pt, qd, np_src, np_out = NARROW[src]
    rng = np.random.default_rng(len(src) * 7 + pt)
    pages = []
    for k in range(30):
        n = int(rng.integers(0, 2000))
        if np_src == np.float16:
            vals = rng.normal(size=n).astype(np.float16) * np.float16(100)
            vals[rng.random(n) < 0.02] = np.nan
        else:
            info = np.iinfo(np_src)
            vals = rng.integers(info.min, int(info.max) + 1, n).astype(np_src)
        mask = rng.random(n) < rng.choice([0.0, 0.1, 0.6])
        p = encode_page(vals, mask, ["plain", "packed", "slotted"][k % 3], pad=int(rng.choice([1, 8])))
        if k % 5 == 4:  # cut short
            p = Page(p.buf[:int(rng.integers(0, len(p.buf) + 1))], p.row_count, p.null_count, p.data_offset)
        pages.append(p)
    t = ctx.table_from_pages([("c", qd, pages, pt)])
    vals, nulls = t.read_column("c")
    want = decode_column_pages(as_tuples(pages), src)
    assert len(vals) == len(want)
    wn = np.array([w is None for w in want], dtype=bool)
    assert np.array_equal(nulls, wn)
    wv = np.array([0 if w is None else w for w in want], dtype=np.float64).astype(np_out)
    if np_out in (np.float32, np.float64):
        nan = np.isnan(wv)
        assert np.array_equal(np.isnan(vals), nan)
        vals, wv = vals[~nan], wv[~nan]
    assert np.array_equal(vals.view(np.uint8), wv.view(np.uint8))
    t.close()
    # a page type widens into one dtype only
    with pytest.raises(A.QmError) as e:
        ctx.table_from_pages([("c", A.QM_I64, pages, pt)])
    assert e.value.status == A.QM_ERR_INVALID


def test_uint32_pages_sum_exactly(ctx):
    """uint32 page values are JS numbers in the reference's operator path
    (decodePlainValues, src/parquet-decode.ts:280-386), so their SUM is a
    float64 sum; values near 2^32 over many rows push every group's sum far
    past 2^32 and stay exact below 2^53, bit for bit against the oracle."""
    rng = np.random.default_rng(77)
    n = 400_000
    vals = rng.integers(4_000_000_000, 4_294_967_296, n, dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 7, n).astype(np.int32)
    t = ctx.table_from_pages([("c", A.QM_F64, encode_column(vals, None, 10_000), A.QM_PT_UINT32),
                              ("k", A.QM_I32, encode_column(key, None, 10_000))])
    q = QueryDescriptor(group_by=["k"], aggregates=[AggregateOp("sum", "c"), AggregateOp("min", "c"),
                                                    AggregateOp("max", "c"), AggregateOp("count", "*")])
    got = t.run(q)
    ref = oracle.run({"c": vals.astype(np.float64), "k": key}, q)
    assert_same(got, ref, rel_tol=0.0)
    sums = got.column("sum_c").values
    assert (sums > 2.0 ** 32).all() and np.array_equal(sums, np.floor(sums))
    t.close()
