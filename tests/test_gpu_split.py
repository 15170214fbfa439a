"""(query, node) work items in the range traversal: with a tiny hand-over
threshold every query past it gives its older pending subtrees to the next
launch, whose CTAs share them out; the counts (added atomically) equal the
counts without any hand-over and the oracle's brute force, for L2, edit
distance (short query strings: the heavy, uneven case) and the stream
update's time-stamped counts."""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu


def test_handed_over_range_counts_equal_brute_force(oracle):
    rows = G.gmm_rows(30000, 32, 16, 0.3, seed=111)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(30000, 2000, seed=112)
    with gts.Index(rows, 2, max_h=4) as idx:
        for frac in (0.001, 0.02):
            r = float(np.float32(G.quantile_radius(2, frac, 20000, 113, rows=rows)))
            idx.plain_split(0)
            whole = idx.range(q, r)
            before = idx.plain_split(64)
            split = idx.range(q, r)
            assert idx.plain_split() > before        # items were handed over
            np.testing.assert_array_equal(split, whole)
            np.testing.assert_array_equal(split, oracle.range_brute(ds, q, r))


def test_handed_over_edit_distance_counts(oracle):
    strs, lens = G.word_strings(40000, seed=114)
    ds = oracle.Dataset(6, strs=strs, lens=lens)
    # the shortest strings as queries: their radius-3 balls hold thousands
    short = np.argsort(lens, kind="stable")[:40].astype(np.int32)
    q = np.concatenate([short, G.query_ids(40000, 200, seed=115)])
    with gts.Index(None, 6, strs=strs, lens=lens, max_h=4) as idx:
        for r in (1.0, 3.0):
            idx.plain_split(0)
            whole = idx.range(q, r)
            before = idx.plain_split(256)
            split = idx.range(q, r)
            np.testing.assert_array_equal(split, whole)
            np.testing.assert_array_equal(split, oracle.range_brute(ds, q, r))
        assert idx.plain_split() > before


def test_handed_over_update_counts():
    rows = G.gmm_rows(6000, 16, 8, 0.3, seed=116)
    flags, ids = G.update_stream(6000, 3000, seed=117, max_in_size=10)
    r = float(np.float32(G.quantile_radius(2, 0.02, 20000, 118, rows=rows)))
    with gts.Index(rows, 2, max_h=3) as a, gts.Index(rows, 2, max_h=3) as b:
        a.plain_split(0)
        b.plain_split(32)
        want, _, _ = a.update_run(flags, ids, r)
        got, _, _ = b.update_run(flags, ids, r)
        np.testing.assert_array_equal(got, want)
        assert b.plain_split() > 0
