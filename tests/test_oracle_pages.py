"""The scan-page decode restatement (oracle/pages.py) pinned on the
reference's known answers for decodePage (src/decode.test.ts:11-99: the
int32, float32, int64 and null-bitmap pages) and on the cases its branches
define (Lance v2 slots, short pages, rowCount 0)."""
import struct

import pytest

from oracle.pages import decode_column_pages, decode_page


def test_int32_page():  # src/decode.test.ts:11-20
    assert decode_page(struct.pack("<3i", 100, -50, 0), "int32") == [100, -50, 0]


def test_float32_page():  # src/decode.test.ts:35-45
    v = decode_page(struct.pack("<2f", 3.14, -2.718), "float32")
    assert len(v) == 2 and v[0] == pytest.approx(3.14, abs=5e-3) and v[1] == pytest.approx(-2.718, abs=5e-3)


def test_int64_page():  # src/decode.test.ts:91-99 (beyond 2^53 stays exact)
    assert decode_page(struct.pack("<2q", 9007199254740993, -42), "int64") == [9007199254740993, -42]


def test_int32_page_with_null_bitmap():  # src/decode.test.ts:77-89
    buf = bytes([0x05]) + struct.pack("<2i", 100, 300)
    assert decode_page(buf, "int32", 1, 3) == [100, None, 300]


def test_lance_v2_slots():
    # bitmap 0b1101 (row 1 NULL), 7 bytes of padding, then a slot per row
    buf = bytes([0x0D]) + bytes(7) + struct.pack("<4q", 10, 99, 30, 40)
    assert decode_page(buf, "int64", 1, 4, 8) == [10, None, 30, 40]
    # slots cut short: only the rows whose slot is there
    assert decode_page(buf[:8 + 16], "int64", 1, 4, 8) == [10, None]
    # offset past the end: no rows
    assert decode_page(buf, "int64", 1, 4, 64) == []


def test_short_and_degenerate_pages():
    # bitmap shorter than ceil(rowCount/8): no rows
    assert decode_page(bytes([0xFF]), "int32", 1, 9) == []
    # packed values run out: present rows past them are NULL
    buf = bytes([0x07]) + struct.pack("<i", 5)
    assert decode_page(buf, "int32", 1, 4) == [5, None, None, None]
    # nullCount above rowCount: no values, every row NULL
    assert decode_page(bytes([0x03]) + struct.pack("<2i", 1, 2), "int32", 5, 2) == [None, None]
    # rowCount 0: every whole value the bytes hold; nullCount ignored
    assert decode_page(struct.pack("<3i", 1, 2, 3) + b"\x01", "int32", 2, 0) == [1, 2, 3]
    # rowCount caps the values; a trailing partial value is dropped
    assert decode_page(struct.pack("<3i", 1, 2, 3), "int32", 0, 2) == [1, 2]
    assert decode_page(struct.pack("<d", 1.5) + b"\x00" * 7, "float64") == [1.5]
    # dataOffsetInPage without NULLs: values from byte 0
    assert decode_page(struct.pack("<2i", 7, 8), "int32", 0, 2, 4) == [7, 8]


def test_pages_concatenate():
    pages = [(struct.pack("<2i", 1, 2), 2, 0, None, False),
             (bytes([0x02]) + struct.pack("<i", 9), 2, 1, None, False),
             (b"", 0, 0, None, False)]
    assert decode_column_pages(pages, "int32") == [1, 2, None, 9]


def test_narrow_page_types():
    # src/decode.test.ts:66-75: float16 0x3C00 reads as 1.0; and the other
    # narrow types of decodePlainValues, little-endian
    assert decode_page(struct.pack("<H", 0x3C00), "float16") == [1.0]
    assert decode_page(struct.pack("<3e", -2.5, 0.0, 65504.0), "float16") == [-2.5, 0.0, 65504.0]
    assert decode_page(bytes([0x80, 0x7F, 0xFF]), "int8") == [-128, 127, -1]
    assert decode_page(bytes([0x80, 0x7F, 0xFF]), "uint8") == [128, 127, 255]
    assert decode_page(struct.pack("<2h", -32768, 7), "int16") == [-32768, 7]
    assert decode_page(struct.pack("<2H", 65535, 7), "uint16") == [65535, 7]
    assert decode_page(struct.pack("<I", 4294967295), "uint32") == [4294967295]
    # with a validity bitmap, packed
    assert decode_page(bytes([0x05]) + bytes([3, 200]), "uint8", 1, 3) == [3, None, 200]
