"""Comparison of a result against the oracle's, with the tolerances of the
path: keys, COUNT, integer SUM/MIN/MAX and float MIN/MAX bit-exact (float
-0 vs 0 included); float SUM/AVG within 1e-12 relative.

For a float SUM whose terms cancel (mixed signs), a relative error against
the reference's own rounded sequential sum is ill-conditioned, so the check
falls back to |gpu - ref| <= 1e-12 * sum|x| together with
|gpu - exact| <= 1e-12 * sum|x| (exact = the oracle's 113-bit sum)."""
from __future__ import annotations

import numpy as np

from querymode_b200 import _abi as A

REL_TOL = 1e-12


def _float_bits_equal(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))


def assert_same(gpu, ref, ordered: bool = True, rel_tol: float = REL_TOL, ctx_msg: str = ""):
    assert gpu.names == ref.names, f"{ctx_msg} columns {gpu.names} != {ref.names}"
    assert gpu.n_rows == ref.n_rows, f"{ctx_msg} rows {gpu.n_rows} != {ref.n_rows}"
    n = gpu.n_rows
    perm = np.arange(n)
    if not ordered and n:
        # align rows by key
        gk = [c for c in gpu.columns if c.is_key]
        rk = [c for c in ref.columns if c.is_key]
        def order(cols):
            keys = []
            for c in reversed(cols):
                v = c.values.view(np.int64) if c.values.dtype == np.float64 else c.values
                keys.append(v)
                if c.nulls is not None:
                    keys.append(c.nulls)
            return np.lexsort(keys) if keys else np.arange(n)
        gperm, rperm = order(gk), order(rk)
    else:
        gperm = rperm = perm
    for g, r in zip(gpu.columns, ref.columns):
        assert g.dtype == r.dtype, f"{ctx_msg} {g.name}: dtype {g.dtype} != {r.dtype}"
        gv, rv = g.values[gperm], r.values[rperm]
        gn = g.nulls[gperm] if g.nulls is not None else np.zeros(n, bool)
        rn = r.nulls[rperm] if r.nulls is not None else np.zeros(n, bool)
        assert np.array_equal(gn, rn), f"{ctx_msg} {g.name}: NULL positions differ"
        live = ~rn
        if g.dtype == A.QM_F64 and not g.is_key and (g.name.startswith("sum_") or g.name.startswith("avg_")
                                                      or g.name in getattr(ref, "diag", {})):
            _assert_float_sum(g.name, gv[live], rv[live], ref, rperm[live], rel_tol, ctx_msg)
        elif g.dtype == A.QM_F64:
            ok = _float_bits_equal(gv[live], rv[live])
            assert ok.all(), f"{ctx_msg} {g.name}: {np.count_nonzero(~ok)} values differ, first " \
                             f"{gv[live][~ok][:3]} vs {rv[live][~ok][:3]}"
        else:
            ok = (gv[live] == rv[live]).reshape(len(gv[live]), -1).all(axis=1) if len(gv[live]) else np.array([], bool)
            assert ok.all(), f"{ctx_msg} {g.name}: {np.count_nonzero(~ok)} values differ, first " \
                             f"{gv[live][~ok][:3]} vs {rv[live][~ok][:3]}"


def _assert_float_sum(name, g, r, ref, ridx, rel_tol, ctx_msg):
    both_nan = np.isnan(g) & np.isnan(r)
    same_inf = np.isinf(g) & (g == r)
    err = np.abs(g - r)
    scale = np.abs(r)
    ok = both_nan | same_inf | (err <= rel_tol * scale)
    diag = getattr(ref, "diag", {}).get(name)
    if diag is not None and not ok.all():
        xhi, xlo, absum = (d[ridx] for d in diag)
        exact = xhi + xlo
        ok2 = (err <= rel_tol * absum) & (np.abs(g - exact) <= rel_tol * absum)
        ok = ok | ok2
    assert ok.all(), (f"{ctx_msg} {name}: {np.count_nonzero(~ok)} of {len(g)} beyond {rel_tol} "
                      f"(worst rel {np.max(err[~ok] / np.maximum(scale[~ok], 1e-300)):.3e}; "
                      f"first {g[~ok][:3]} vs {r[~ok][:3]})")
