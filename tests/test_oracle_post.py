"""The oracle's restatement of the reference's post-aggregate operators
(TopKOperator heap, InMemorySortOperator, LimitOperator), pinned to the
reference's own TopK test and to cases worked by hand."""
import math

import numpy as np

from oracle.post import limit_order, sort_order, topk_order
from querymode_b200 import datagen


def test_topk_generate_rows_matches_reference_test():
    # src/operators-conformance.test.ts:576-593: TopK(amount DESC, 100) over
    # generateRows has the same amounts as ORDER BY amount DESC LIMIT 100
    vals = [int(x) for x in datagen.generate_rows(200_000)["amount"]]
    out = topk_order(vals, True, 100, 0)
    assert sorted((vals[i] for i in out), reverse=True) == sorted(vals, reverse=True)[:100]
    assert [vals[i] for i in out] == sorted((vals[i] for i in out), reverse=True)


def test_topk_ties_follow_the_heap():
    # k = 2 ascending over [5, 5, 1]: the heap root is row 0 (the siftUp of
    # row 1 stops on a tie), so row 2 evicts row 0 and the result is [2, 1]
    assert topk_order([5, 5, 1], False, 2, 0) == [2, 1]
    # all equal: nothing replaces the root; extraction takes 0, then moves the
    # last entry to the root: [0, 2, 1], reversed
    assert topk_order([7, 7, 7, 7], False, 3, 0) == [1, 2, 0]


def test_nulls_and_nan_last_both_directions():
    vals = [3.0, None, math.nan, -0.0, 0.0, 2.5, None]
    assert sort_order(vals, False, 0) == [3, 4, 5, 0, 1, 2, 6]
    assert sort_order(vals, True, 0) == [0, 5, 3, 4, 1, 2, 6]
    assert topk_order(vals, True, 3, 0) == [0, 5, 3]
    # ascending k = 3 (LIMIT 2 OFFSET 1): the heap ends as [5, 4, 3] and
    # extracts 5, 3, 4 (-0 and 0 tie); reversed [4, 3, 5], sliced past 1 row
    assert topk_order(vals, False, 2, 1) == [3, 5]


def test_limit_offset_slices():
    assert limit_order(10, 3, 0) == [0, 1, 2]
    assert limit_order(10, 3, 8) == [8, 9]
    assert limit_order(10, None, 7) == [7, 8, 9]
    assert limit_order(10, 0, 2) == []
    assert sort_order([2, 1, 3], False, 5) == []


def test_topk_values_are_the_k_best():
    rng = np.random.default_rng(0)
    for _ in range(50):
        n = int(rng.integers(1, 300))
        vals = [int(v) for v in rng.integers(0, 20, n)]
        k = int(rng.integers(0, 40))
        desc = bool(rng.integers(0, 2))
        out = topk_order(vals, desc, k, 0)
        best = sorted(vals, reverse=desc)[:k]
        assert [vals[i] for i in out] == best
