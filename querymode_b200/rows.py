"""Result columns -> Row[] the way finalizePartialAgg emits them
(src/partial-agg.ts:306-352).

Values map JS -> Python as: number -> float (int for COUNT and for integer
MIN/MAX, whose JS numbers are exact integers), bigint -> int, null -> None.
Group keys are restored exactly (an int64 key is a JS number when it
round-trips through String, else a bigint; both are exact Python ints).

Reference quirks kept on purpose:
  * an ungrouped aggregate always yields one row, NULLs for SUM/AVG/MIN/MAX of
    an empty input and 0 for COUNT (src/partial-agg.ts:313-320, :109-111);
  * a GROUP BY that matches no row yields ``[{}]`` — one empty row — because
    finalizePartialAgg falls into its ungrouped branch with no states
    (src/partial-agg.ts:313-320 reached from src/operators.ts:1679-1680).
"""
from __future__ import annotations

from typing import Any

from .engine import Result


def result_to_rows(result: Result, grouped: bool) -> list[dict[str, Any]]:
    if grouped and result.n_rows == 0:
        return [{}]
    cols = [(c.name, c.pyvalues()) for c in result.columns]
    return [{name: vals[i] for name, vals in cols} for i in range(result.n_rows)]
