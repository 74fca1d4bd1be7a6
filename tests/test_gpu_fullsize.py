"""The measured workloads at their full sizes against the oracle.

The bench times these queries at these sizes; here the device results are
compared with the reference's one-batch result (oracle.run_full: every
group's rows summed in row order, groups in first-seen order) with the
path's tolerances (tests/helpers.py): keys, first-seen order, COUNT, integer
SUM, float MIN / MAX bit-exact; float SUM / AVG within 1e-12 relative.

At these sizes the group tables leave L2, the 16.7M-group aggregate runs in
key-range passes, and int32 sums switch accumulator width on the row count
(src/partial-agg.ts:225-352 merge and finalize; the at-scale conformance
pattern of src/operators-conformance.test.ts:408-447).
"""
import numpy as np
import pytest

import oracle
from querymode_b200 import datagen
from tests.helpers import assert_same

pytestmark = pytest.mark.gpu


def test_events_100m_full(ctx):
    """events_100m: 100M rows, key int64 Zipf(1.1) over 65,536 values, the
    30-day window AND qty > 10 query (seed 1, the bench's table)."""
    cols = datagen.events(100_000_000, seed=1)
    q = datagen.events_query()
    t = ctx.table(cols)
    g = t.run(q)
    t.close()
    r = oracle.run_full(cols, q)
    assert g.n_rows > 60_000
    assert g.stats.rows_selected == int(r.column("count_*").values.sum())
    assert_same(g, r, ctx_msg="events_100m")


@pytest.fixture(scope="module")
def wide_200m():
    return datagen.wide_keys(200_000_000, seed=2, n_keys=1 << 24)


@pytest.mark.parametrize("filtered", [True, False], ids=["filtered", "unfiltered"])
def test_wide_keys_200m_full(ctx, wide_200m, filtered):
    """wide_keys_200m: 200M rows, key int64 uniform over 2^24 values;
    flag = 1 AND val > 0 (~0.5 % selected) and the unfiltered 16.7M-group
    aggregate."""
    q = datagen.wide_keys_query(filtered)
    t = ctx.table(wide_200m)
    g = t.run(q)
    t.close()
    r = oracle.run_full(wide_200m, q)
    if not filtered:
        assert g.n_rows > 16_000_000
        assert g.stats.rows_selected == 200_000_000
    assert_same(g, r, ctx_msg=f"wide_keys_200m filtered={filtered}")


def test_orders_1m_seed0_matches_whole_table_sum(ctx):
    """orders_1m (seed 0): the counts of every group add up to the selected
    rows, and the one-batch oracle agrees."""
    cols = datagen.orders()
    t = ctx.table(cols)
    g = t.run(datagen.orders_query())
    t.close()
    r = oracle.run_full(cols, datagen.orders_query())
    assert_same(g, r)
    assert int(np.sum(g.column("count_*").values)) == int((cols["status"] == 1).sum())
