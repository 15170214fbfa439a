"""Every benchmark configuration's shape at a reduced but non-trivial size,
checked against the oracle's exact brute force (the reference's per-site
arithmetic) on a sample of queries:

* 50,000 x 300 L2 (the first configuration at full size): kNN k = 8 in
  both forms (the tensor-core one streams K above dim 128) and range counts
  at the 0.1 % distance quantile;
* 200,000 strings, edit distance: range r = 1, 2, 3 (short query strings
  included: the heavy, uneven queries) and kNN k = 16;
* 200,000 x 128 L2: kNN with k over {1, 8, 32, 64}, fast and plain;
* 1,000,000 two-dimensional L1 hotspot points: range counts at the 0.01 %
  quantile;
* 100,000 x 300 L2 stream update (copy inserts and new-row inserts).
"""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu


def test_gmm50k_d300(oracle):
    rows = G.gmm_rows(50_000, 300, 64, 0.3, seed=201)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(50_000, 200, seed=202)
    r = float(np.float32(G.quantile_radius(2, 0.001, 200_000, 203, rows=rows)))
    with gts.Index(rows, 2, max_h=5) as idx:
        bk, bi, _ = oracle.knn_brute(ds, q, 8)
        for form in (gts.FORM_FAST, gts.FORM_PLAIN):
            kth, ids, _ = idx.knn(q, 8, form=form, return_ids=True)
            np.testing.assert_array_equal(ids, bi, err_msg=f"form {form}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"form {form}")
        want = oracle.range_brute(ds, q, r)
        np.testing.assert_array_equal(idx.range(q, r, form=gts.FORM_FAST), want)
        np.testing.assert_array_equal(idx.range(q, r), want)


def test_words200k_edit(oracle):
    strs, lens = G.word_strings(200_000, seed=204)
    ds = oracle.Dataset(6, strs=strs, lens=lens)
    short = np.argsort(lens, kind="stable")[:20].astype(np.int32)
    q = np.concatenate([short, G.query_ids(200_000, 100, seed=205)])
    with gts.Index(None, 6, strs=strs, lens=lens, max_h=5) as idx:
        for r in (1.0, 2.0, 3.0):
            np.testing.assert_array_equal(idx.range(q, r), oracle.range_brute(ds, q, r), err_msg=f"r={r}")
        kth, ids, _ = idx.knn(q, 16, return_ids=True)
        bk, bi, _ = oracle.knn_brute(ds, q, 16)
        np.testing.assert_array_equal(kth, bk)
        np.testing.assert_array_equal(ids, bi)


def test_gmm200k_d128_kmix(oracle):
    rows = G.gmm_rows(200_000, 128, 256, 0.2, seed=206)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(200_000, 300, seed=207)
    with gts.Index(rows, 2, max_h=5) as idx:
        for k in (1, 8, 32, 64):
            bk, bi, _ = oracle.knn_brute(ds, q, k)
            for form in (gts.FORM_FAST, gts.FORM_PLAIN):
                kth, ids, _ = idx.knn(q, k, form=form, return_ids=True)
                np.testing.assert_array_equal(ids, bi, err_msg=f"k={k} form {form}")
                np.testing.assert_array_equal(kth, bk, err_msg=f"k={k} form {form}")


def test_hotspots1m_l1(oracle):
    rows = G.hotspot_points(1_000_000, seed=208)
    ds = oracle.Dataset(1, rows)
    q = G.query_ids(1_000_000, 500, seed=209)
    r = float(np.float32(G.quantile_radius(1, 0.0001, 2_000_000, 210, rows=rows)))
    with gts.Index(rows, 1, max_h=6) as idx:
        np.testing.assert_array_equal(idx.range(q, r), oracle.range_brute(ds, q, r))


def test_gmm100k_d300_update_streams(oracle):
    rows = G.gmm_rows(100_000, 300, 64, 0.3, seed=211)
    ds = oracle.Dataset(2, rows)
    r = float(np.float32(G.quantile_radius(2, 0.001, 200_000, 212, rows=rows)))
    flags, ids = G.update_stream(100_000, 1500, seed=213, max_in_size=10)
    want = oracle.update_run(ds, oracle.params(max_h=5), 10, flags, ids, r, exact=True)
    with gts.Index(rows, 2, max_h=5, max_in_size=10) as idx:
        got, _, _ = idx.update_run(flags, ids, r)
    np.testing.assert_array_equal(got, want)
    flags, ids = G.update_stream_new_rows(100_000, 1500, seed=214, max_in_size=10)
    new_rows = G.gmm_rows(int((flags == 0).sum()), 300, 64, 0.3, seed=215)
    want = oracle.update_run_rows(ds, 10, flags, ids, new_rows, r)
    with gts.Index(rows, 2, max_h=5, max_in_size=10) as idx:
        got, _, _ = idx.update_run_rows(flags, ids, new_rows, r)
    np.testing.assert_array_equal(got, want)
