"""Scan pages in the layouts the reference's decodePage reads (src/decode.ts:251-331),
written from numpy arrays: plain values, a validity bitmap (bit set = a value)
followed by the packed non-NULL values, or a bitmap padded to an alignment
followed by one slot per row (Lance v2 nullable pages)."""
import numpy as np

from querymode_b200.engine import Page


def encode_page(vals: np.ndarray, mask, mode: str, pad: int = 8) -> Page:
    n = len(vals)
    if mode == "plain" or mask is None or not mask.any():
        return Page(vals.tobytes(), n, 0)
    bitmap = np.packbits(~mask, bitorder="little").tobytes()
    if mode == "packed":
        return Page(bitmap + vals[~mask].tobytes(), n, int(mask.sum()))
    off = -(-len(bitmap) // pad) * pad
    slots = vals.copy()
    slots[mask] = 0
    return Page(bitmap + bytes(off - len(bitmap)) + slots.tobytes(), n, int(mask.sum()), off)


def encode_column(vals: np.ndarray, mask, rows_per_page: int, modes=("packed",), rng=None) -> list:
    pages = []
    for k, a in enumerate(range(0, len(vals), rows_per_page)):
        m = None if mask is None else mask[a:a + rows_per_page]
        mode = modes[k % len(modes)] if rng is None else modes[rng.integers(len(modes))]
        pages.append(encode_page(vals[a:a + rows_per_page], m, mode))
    return pages


def as_tuples(pages: list) -> list:
    """(buf, row_count, null_count, data_offset, parquet) for oracle/pages.py."""
    return [(bytes(p.buf), p.row_count, p.null_count, p.data_offset, p.parquet) for p in pages]
