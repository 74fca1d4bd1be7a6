"""Test infrastructure: the reference's Parquet column-chunk decode restated
for PLAIN numeric pages, to check the device decoder against.

Follows src/parquet-decode.ts: decodeParquetColumnChunk (:390-618, the
DATA_PAGE v1 and v2 PLAIN paths, the v1 level-section heuristic),
parsePageHeader / parseDataPageHeader(V2) (:204-276, Thrift compact
protocol), readV1DefLevels (:108-116), decodeRleBitPacked (:119-188) and
decodePlainValues (:280-386).  Values come back as Python numbers (int64 as
int, like the reference's bigint) with None for NULL.
"""
from __future__ import annotations

import struct


class _Thrift:
    """Thrift compact protocol with the reference's reading rules
    (ThriftReader, src/parquet.ts:44-183): varints of at most 5 bytes keep
    the low 32 bits, i32 fields are their zigzag as an int32, the buffer's
    end ends a struct, unknown types take no bytes."""

    def __init__(self, b: bytes, pos: int):
        self.b, self.pos, self.last, self.stack = b, pos, 0, []

    def byte_at(self, i: int) -> int:
        return self.b[i] if i < len(self.b) else 0  # JS reads undefined: 0 in bit operations

    def varint(self) -> int:
        v = shift = 0
        while self.pos < len(self.b):
            c = self.b[self.pos]
            self.pos += 1
            v = (v | ((c & 0x7F) << shift)) & 0xFFFFFFFF
            if not c & 0x80:
                return v
            shift += 7
            if shift >= 35:
                return v
        return v

    def zigzag(self) -> int:
        v = self.varint()
        r = (v >> 1) ^ (-(v & 1) & 0xFFFFFFFF)
        return r - (1 << 32) if r & 0x80000000 else r

    def field(self):
        if self.pos >= len(self.b):
            return None
        h = self.b[self.pos]
        self.pos += 1
        if h == 0:
            return None
        t, d = h & 0x0F, h >> 4
        fid = self.last + d if d else self.zigzag()
        self.last = fid
        return fid, t

    def skip(self, t: int, depth: int = 0):
        if depth > 64:
            return
        if t == 3:
            self.pos += 1
        elif t in (4, 5):
            self.varint()
        elif t == 6:
            while self.pos < len(self.b):
                c = self.b[self.pos]
                self.pos += 1
                if not c & 0x80:
                    break
        elif t == 7:
            self.pos += 8
        elif t == 8:
            n = self.varint()
            self.pos += n
        elif t in (9, 10):
            h = self.byte_at(self.pos)
            self.pos += 1
            size = h >> 4
            if size == 15:
                size = self.varint()
            i = 0
            # past the buffer's end only the position changes, and it is past
            # already; elements of no bytes (bools, unknown types) change nothing
            while i < size and self.pos < len(self.b) and 3 <= (h & 0x0F) <= 12:
                self.skip(h & 0x0F, depth + 1)
                i += 1
        elif t == 11:
            size = self.varint()
            if size:
                kv = self.byte_at(self.pos)
                self.pos += 1
                i = 0
                while i < size and self.pos < len(self.b) and (3 <= kv >> 4 <= 12 or 3 <= (kv & 0x0F) <= 12):
                    self.skip(kv >> 4, depth + 1)
                    self.skip(kv & 0x0F, depth + 1)
                    i += 1
        elif t == 12:
            self.stack.append(self.last)
            self.last = 0
            while (f := self.field()) is not None:
                self.skip(f[1], depth + 1)
            self.last = self.stack.pop()


def parse_page_header(b: bytes, offset: int) -> dict:
    r = _Thrift(b, offset)
    h = dict(type=0, uncompressed=0, compressed=0, num_values=0, encoding=0, def_len=0, rep_len=0)
    while (f := r.field()) is not None:
        fid, t = f
        if fid == 1:
            h["type"] = r.zigzag()
        elif fid == 2:
            h["uncompressed"] = r.zigzag()
        elif fid == 3:
            h["compressed"] = r.zigzag()
        elif fid in (5, 7, 8):
            r.stack.append(r.last)
            r.last = 0
            while (g := r.field()) is not None:
                gid, gt = g
                if gid == 1:
                    h["num_values"] = r.zigzag()
                elif fid != 8 and gid == 2:
                    h["encoding"] = r.zigzag()
                elif fid == 8 and gid == 4:
                    h["encoding"] = r.zigzag()
                elif fid == 8 and gid == 5:
                    h["def_len"] = r.zigzag()
                elif fid == 8 and gid == 6:
                    h["rep_len"] = r.zigzag()
                elif fid == 8 and gid in (2, 3):
                    r.zigzag()  # num_nulls, num_rows: read as i32 whatever their type
                elif fid == 8 and gid == 7:
                    pass  # is_compressed: in the type nibble
                else:
                    r.skip(gt)
            r.last = r.stack.pop()
        else:
            r.skip(t)
    h["header_size"] = r.pos - offset
    return h


def _run_varint(b: bytes, pos: int) -> tuple[int, int]:
    """readVarint (src/footer.ts:183-200): to the terminator or the end, the
    low 32 bits."""
    v = shift = 0
    while pos < len(b):
        c = b[pos]
        pos += 1
        if shift < 32:
            v = (v | ((c & 0x7F) << shift)) & 0xFFFFFFFF
        if not c & 0x80:
            break
        shift += 7
    return v, pos


def decode_rle_bit_packed(b: bytes, bit_width: int, max_values: int) -> list[int]:
    """decodeRleBitPacked (src/parquet-decode.ts:119-188).  A run's count is
    its header shifted as a signed 32-bit number (the reference's
    `header >> 1`); a negative bit-packed count, after which the reference
    would step back and read the same bytes again without end, ends the
    stream."""
    values: list[int] = []
    pos = 0
    mask = (1 << bit_width) - 1
    while pos < len(b) and len(values) < max_values:
        header, pos = _run_varint(b, pos)
        half = (header - (1 << 32) if header & 0x80000000 else header) >> 1
        if header & 1 == 0:
            val = 0
            for i in range((bit_width + 7) // 8):
                if pos < len(b):
                    val |= b[pos] << (8 * i)
                    pos += 1
            values += [val & mask] * max(0, min(half, max_values - len(values)))
        else:
            if half < 0:
                break
            groups = half
            n = min(groups * 8, max_values - len(values))
            bitpos = pos * 8
            for _ in range(n):
                v = 0
                for k in range(bit_width):
                    byte = bitpos >> 3
                    bit = (b[byte] >> (bitpos & 7)) & 1 if byte < len(b) else 0
                    v |= bit << k
                    bitpos += 1
                values.append(v)
            pos += (groups * 8 * bit_width + 7) // 8
    return values


_FMT = {"int32": ("<i", 4), "int64": ("<q", 8), "float32": ("<f", 4), "float64": ("<d", 8),
        # narrower page types of decodePlainValues (src/parquet-decode.ts:288-348); float16 as its exact value
        "int8": ("<b", 1), "uint8": ("<B", 1), "int16": ("<h", 2), "uint16": ("<H", 2), "uint32": ("<I", 4),
        "float16": ("<e", 2)}


def decode_plain(b: bytes, dtype: str, n: int) -> list:
    fmt, w = _FMT[dtype]
    n = min(n, len(b) // w)
    return [struct.unpack_from(fmt, b, i * w)[0] for i in range(n)]


def _dict_bit_width(n: int) -> int:
    """ceil(log2(n)) as the reference computes it (0 for n <= 1)."""
    return 0 if n <= 1 else (n - 1).bit_length()


def decode_column_chunk(b: bytes, dtype: str, num_values: int) -> list:
    """decodeParquetColumnChunk (src/parquet-decode.ts:390-618) for an
    uncompressed chunk: dictionary pages, v1 / v2 data pages, PLAIN values or
    RLE_DICTIONARY / RLE (encodings 8 and 3) indices into the dictionary."""
    values: list = []
    w = _FMT[dtype][1]
    dictionary = None
    pos = 0
    while pos < len(b) and len(values) < num_values:
        h = parse_page_header(b, pos)
        if h["compressed"] <= 0:
            break
        pos += h["header_size"]
        page = b[pos:pos + h["compressed"]]
        pos += h["compressed"]
        if h["type"] == 2:  # DICTIONARY_PAGE
            dictionary = decode_plain(page, dtype, h["num_values"])
            continue
        if h["type"] not in (0, 3):
            continue
        enc = h["encoding"]
        is_dict = enc in (8, 3)
        if not is_dict and enc != 0:
            raise NotImplementedError("encoding %d" % enc)
        defs = None
        off = 0
        if h["type"] == 0:
            if 8 <= len(page):
                plen = struct.unpack_from("<i", page, 0)[0]
                max_def = max(64, -(-h["num_values"] // 4) + 8)
                if 0 < plen <= max_def and plen < len(page) - 4:
                    if is_dict and dictionary is not None:
                        after = 4 + plen
                        level = after < len(page) and page[after] == _dict_bit_width(len(dictionary))
                    else:
                        rem = len(page) - 4 - plen
                        level = 0 <= rem <= h["num_values"] * w
                    if level:
                        defs = decode_rle_bit_packed(page[4:4 + plen], 1, h["num_values"])
                        off = 4 + plen
        else:
            d0 = h["rep_len"]
            if h["def_len"] > 0:
                defs = decode_rle_bit_packed(page[d0:d0 + h["def_len"]], 1, h["num_values"])
            off = d0 + h["def_len"]

        def is_null(i):
            return defs is not None and i < len(defs) and defs[i] == 0

        nonnull = h["num_values"] if defs is None else sum(1 for d in defs if d > 0)
        if is_dict:
            if dictionary is None:
                continue
            bw = page[off] if off < len(page) else 0
            if bw == 0:
                first = dictionary[0] if dictionary else None
                for i in range(h["num_values"]):
                    if len(values) >= num_values:
                        break
                    values.append(None if is_null(i) else first)
            else:
                idx = decode_rle_bit_packed(page[off + 1:], bw, nonnull)
                ip = 0
                for i in range(h["num_values"]):
                    if len(values) >= num_values:
                        break
                    if is_null(i):
                        values.append(None)
                    else:
                        k = idx[ip] if ip < len(idx) else 0
                        ip += 1
                        values.append(dictionary[k] if k < len(dictionary) else None)
            continue
        decoded = decode_plain(page[off:], dtype, nonnull)
        if defs is not None:
            dp = 0
            for i in range(h["num_values"]):
                if len(values) >= num_values:
                    break
                if is_null(i):
                    values.append(None)
                else:
                    values.append(decoded[dp] if dp < len(decoded) else None)
                    dp += 1
        else:
            for v in decoded:
                if len(values) >= num_values:
                    break
                values.append(v)
    return values
