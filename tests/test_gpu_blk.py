"""The block-stationary filter (each needed block read once per run and
multiplied with the queries that need it): bit-identical kNN answers and
range counts to exact brute force in the reference's arithmetic, like the
tile filter, including pair-capacity overflow and ties."""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu

CASES = [  # (n, dim, comps, sigma, nq, max_h)
    (20000, 128, 32, 0.2, 300, 5),
    (9000, 64, 16, 0.3, 257, 4),       # ragged query count, n not a multiple of 128
    (7777, 100, 8, 0.25, 130, 4),      # dimension padded to 128
    (4000, 32, 4, 1.0, 129, 4),        # kp 64
    (3000, 128, 1, 0.05, 64, 4),       # one tight cluster: every query needs every block
]


def _pin(idx, k):
    idx.set_fast_config(k, False, 1, 16, by_block=True)
    assert idx.fast_config(k)["by_block"]


@pytest.mark.parametrize("n,dim,comps,sigma,nq,max_h", CASES)
def test_by_block_knn_equals_brute_force(oracle, n, dim, comps, sigma, nq, max_h):
    rows = G.gmm_rows(n, dim, comps, sigma, seed=n + dim)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(n, nq, seed=n + 1)
    with gts.Index(rows, 2, max_h=max_h) as idx:
        for k in (1, 8, 33, 64):
            _pin(idx, k)
            kth, ids, dis = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k}")


def test_by_block_pairs_beyond_capacity_are_answered_again(oracle):
    """A single tight cluster: every query needs most of the 157 blocks, more
    pairs than the run stores (64 per query); the queries whose pairs were not
    stored are marked and answered again (a second filter pass, through the
    tile filter), exactly."""
    rows = G.gmm_rows(20000, 128, 1, 0.05, seed=131)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(20000, 200, seed=132)
    with gts.Index(rows, 2, max_h=4) as idx:
        _pin(idx, 8)
        kth, ids, dis = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)
        assert idx.search_stats()["passes"] >= 2
    bk, bi, bd = oracle.knn_brute(ds, q, 8)
    np.testing.assert_array_equal(ids, bi)
    np.testing.assert_array_equal(kth, bk)
    np.testing.assert_array_equal(dis, bd)


def test_by_block_ties_and_repeated_queries(oracle):
    """Every row twice (equal-distance pairs, ties broken by id) and query ids
    repeated within the batch."""
    base = G.gmm_rows(4000, 64, 10, 0.3, seed=141)
    rows = np.concatenate([base, base])
    ds = oracle.Dataset(2, rows)
    q = np.concatenate([G.query_ids(len(rows), 200, seed=142)] * 2)
    with gts.Index(rows, 2, max_h=4) as idx:
        for k in (2, 7, 16):
            _pin(idx, k)
            kth, ids, dis = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k}")


def test_by_block_equals_tile_filter_and_replays(oracle):
    """The two filters give identical answers on one index; the block
    filter's pass replays from its captured graph."""
    rows = G.gmm_rows(30000, 128, 64, 0.2, seed=151)
    q = G.query_ids(30000, 2500, seed=152)
    with gts.Index(rows, 2, max_h=5) as idx:
        idx.set_fast_config(8, False, 4, 16)
        a = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)
        _pin(idx, 8)
        n0 = idx.fast_graphs()
        for _ in range(2):
            b = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)
        assert idx.fast_graphs() - n0 == 2
        st = idx.search_stats()
        assert st["blocks"] > 0 and st["appended"] > 0


@pytest.mark.parametrize("n,dim,comps,sigma,max_h", [(20000, 128, 32, 0.2, 5), (7777, 100, 8, 0.25, 4),
                                                     (4000, 32, 4, 1.0, 4)])
def test_by_block_range_counts_equal_brute_force(oracle, n, dim, comps, sigma, max_h):
    """Range counts through both filters equal exact brute force, from the
    query alone to radii holding thousands of objects."""
    rows = G.gmm_rows(n, dim, comps, sigma, seed=n + 17)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(n, 300, seed=n + 18)
    with gts.Index(rows, 2, max_h=max_h) as idx:
        for frac in (0.0, 0.001, 0.01, 0.2):
            r = 0.0 if frac == 0 else float(np.float32(G.quantile_radius(2, frac, 20000, n + 19, rows=rows)))
            want = oracle.range_brute(ds, q, r)
            for variant in (0, 1):
                assert idx.fast_range_variant(variant) == variant
                got = idx.range(q, r, form=gts.FORM_FAST)
                np.testing.assert_array_equal(got, want, err_msg=f"r={r} variant={variant}")


def test_by_block_many_items_per_cta_equal_tile_filter():
    """200,000 objects and 6,000 queries: every CTA runs dozens of items, so
    stages, accumulators and header slots are reused many times over; the
    answers equal the tile filter's for small, middle and large k."""
    rows = G.gmm_rows(200000, 64, 128, 0.25, seed=161)
    q = G.query_ids(200000, 6000, seed=162)
    with gts.Index(rows, 2, max_h=6) as idx:
        for k in (1, 8, 64):
            idx.set_fast_config(k, False, 1 if k > 32 else 4, 16)
            a = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            _pin(idx, k)
            b = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            st = idx.search_stats()
            assert st["blocks"] > 20 * 148, st
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y, err_msg=f"k={k}")
