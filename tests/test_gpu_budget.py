"""gts_params.mem_budget_gb bounds a search call's device scratch: under a
small budget the same calls run in more, smaller runs (fast form), chunks
(seeded plain form) or batches (update path) with identical answers, and a
budget below one run is refused with GTS_ERR_NOMEM."""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu


def _pair(rows, budget_gb, **kw):
    return gts.Index(rows, 2, **kw), gts.Index(rows, 2, mem_budget_gb=budget_gb, **kw)


def test_small_budget_fast_knn_and_range_equal_the_default(oracle):
    rows = G.gmm_rows(20000, 32, 16, 0.3, seed=41)
    qids = G.query_ids(20000, 3000, seed=42)
    r = float(np.float32(G.quantile_radius(2, 0.002, 20000, 43, rows=rows)))
    big, small = _pair(rows, 0.004, max_h=4)   # ~4 MB: runs of a few tiles
    with big, small:
        for k in (1, 8, 33):
            kb, ib, db = big.knn(qids, k, form=gts.FORM_FAST, return_ids=True)
            ks, is_, ds = small.knn(qids, k, form=gts.FORM_FAST, return_ids=True)
            np.testing.assert_array_equal(ks, kb)
            np.testing.assert_array_equal(is_, ib)
        np.testing.assert_array_equal(small.range(qids, r, form=gts.FORM_FAST), big.range(qids, r, form=gts.FORM_FAST))
        # the runs are smaller: more filter passes for the same batch
        small.knn(qids, 8, form=gts.FORM_FAST)
        big.knn(qids, 8, form=gts.FORM_FAST)
        assert small.search_stats()["passes"] > big.search_stats()["passes"]
        bk, _, _ = oracle.knn_brute(oracle.Dataset(2, rows), qids[:200], 8)
        np.testing.assert_array_equal(small.knn(qids[:200], 8, form=gts.FORM_FAST), bk)


def test_budget_below_one_run_is_refused():
    rows = G.gmm_rows(5000, 16, 8, 0.3, seed=44)
    with gts.Index(rows, 2, max_h=3, mem_budget_gb=1e-6) as idx:   # about 1 KB
        with pytest.raises(gts.GtsError) as e:
            idx.knn(np.arange(300, dtype=np.int32), 8, form=gts.FORM_FAST)
        assert e.value.code == -3
        with pytest.raises(gts.GtsError) as e:
            idx.range(np.arange(300, dtype=np.int32), 1.0, form=gts.FORM_FAST)
        assert e.value.code == -3
        # the plain traversal needs no scratch: it still answers
        assert len(idx.knn(np.arange(300, dtype=np.int32), 8)) == 300


def test_small_budget_update_stream_equals_the_default():
    rows = G.gmm_rows(4000, 8, 8, 0.3, seed=45)
    flags, ids = G.update_stream(4000, 3000, seed=46, max_in_size=10)
    r = float(np.float32(G.quantile_radius(2, 0.01, 20000, 47, rows=rows)))
    # the stream's entries (16 B each), their offsets and 1 KB stay resident;
    # the budget leaves room for batches of 50 queries (16 B each)
    n_ent = 4000 + int((flags == 0).sum())
    fixed = 4 * 4001 + 16 * n_ent + 1024
    big, small = _pair(rows, (fixed + 16 * 50) / 2**30, max_h=3)
    with big, small:
        want, _, _ = big.update_run(flags, ids, r)
        got, _, _ = small.update_run(flags, ids, r)
        np.testing.assert_array_equal(got, want)
