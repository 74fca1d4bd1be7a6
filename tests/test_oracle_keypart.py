"""The oracle's key-partitioned threaded run (oracle.run_full) against its
single-thread one-batch run: the same groups, first-seen order and every
value bit for bit (float sums included: each group's rows are still summed
in row order)."""
import numpy as np
import pytest

import oracle
from querymode_b200 import datagen
from tests.helpers import assert_same
from tests.test_oracle_jsref import make_table, rand_query


@pytest.mark.parametrize("seed", range(30))
def test_keypart_equals_one_batch(seed):
    rng = np.random.default_rng(900 + seed)
    cols = make_table(rng, n=int(rng.choice([300, 5000, 70000])))
    q = rand_query(rng)
    a = oracle.run(cols, q, batch_rows=0)
    b = oracle.run_full(cols, q, threads=int(rng.integers(2, 9)))
    assert_same(b, a, rel_tol=0.0, ctx_msg=str(q))


def test_keypart_many_groups():
    cols = datagen.wide_keys(400_000, seed=5, n_keys=1 << 17)
    for filtered in (True, False):
        q = datagen.wide_keys_query(filtered)
        assert_same(oracle.run_full(cols, q, threads=7), oracle.run(cols, q), rel_tol=0.0)
