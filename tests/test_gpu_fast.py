"""The fast form (BF16 tensor-core filter + exact recheck): bit-identical
answers to exact brute force in the reference's leaf arithmetic."""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu

CASES = [  # (n, dim, comps, sigma, nq, max_h)
    (20000, 128, 32, 0.2, 300, 5),     # the headline shape, small
    (9000, 64, 16, 0.3, 257, 4),       # ragged query count, n not a multiple of 128
    (7777, 100, 8, 0.25, 130, 4),      # dimension padded to 128 inside the filter
    (4000, 32, 4, 1.0, 129, 4),
    (3000, 128, 1, 0.05, 64, 4),       # one tight cluster: many near-ties
    # above a padded dimension of 128 the filter streams K in 64-wide chunks
    (6000, 300, 16, 0.3, 200, 4),      # the d = 300 configurations' width (kp 320, the limit)
    (5000, 200, 8, 0.3, 130, 4),       # kp 256
    (4000, 129, 8, 0.3, 64, 4),        # one past the resident form (kp 192)
]


@pytest.mark.parametrize("n,dim,comps,sigma,nq,max_h", CASES)
def test_fast_knn_equals_brute_force(oracle, n, dim, comps, sigma, nq, max_h):
    rows = G.gmm_rows(n, dim, comps, sigma, seed=n + dim)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(n, nq, seed=n + 1)
    with gts.Index(rows, 2, max_h=max_h) as idx:
        for k in (1, 8, 33, 64):
            kth, ids, dis = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k}")


def test_fast_equals_plain_and_counts_work():
    rows = G.gmm_rows(30000, 128, 64, 0.2, seed=5)
    q = G.query_ids(30000, 1000, seed=6)
    with gts.Index(rows, 2, max_h=5) as idx:
        a = idx.knn(q, 8, form=gts.FORM_PLAIN, return_ids=True)
        b = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)
        st = idx.search_stats()
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    assert st["objects"] > 0 and st["exact"] >= 8 * len(q)


def test_fast_falls_back_outside_its_shape(oracle):
    """Dimensions above the filter's limit (320) and k above 64 take the plain path."""
    rows = G.gmm_rows(3000, 400, 8, 0.3, seed=7)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(3000, 40, seed=8)
    with gts.Index(rows, 2, max_h=4) as idx:
        kth = idx.knn(q, 8, form=gts.FORM_FAST)
        np.testing.assert_array_equal(kth, oracle.knn_brute(ds, q, 8)[0])
        kth = idx.knn(q, 100, form=gts.FORM_FAST)
        np.testing.assert_array_equal(kth, oracle.knn_brute(ds, q, 100)[0])


def test_fast_batches_larger_than_one_run(oracle):
    """More queries than one filter run holds (32,768) are answered in
    consecutive runs over the same scratch; repeated query ids included."""
    rows = G.gmm_rows(6000, 16, 12, 0.3, seed=11)
    ds = oracle.Dataset(2, rows)
    q = np.random.default_rng(12).integers(0, 6000, size=40000).astype(np.int32)
    with gts.Index(rows, 2, max_h=4) as idx:
        kth, ids, dis = idx.knn(q, 5, form=gts.FORM_FAST, return_ids=True)
    bk, bi, bd = oracle.knn_brute(ds, q, 5)
    np.testing.assert_array_equal(ids, bi)
    np.testing.assert_array_equal(kth, bk)
    np.testing.assert_array_equal(dis, bd)


def test_autotuner_picks_a_config_and_stays_exact(oracle):
    """The first batch of >= 2048 queries for a k times every candidate
    configuration (all exact) and keeps the fastest; later calls use it."""
    rows = G.gmm_rows(30000, 64, 24, 0.25, seed=21)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(30000, 2500, seed=22)
    with gts.Index(rows, 2, max_h=5) as idx:
        assert not idx.fast_config(8)["tuned"]
        kth, ids, _ = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)
        cfg = idx.fast_config(8)
        assert cfg["tuned"] and cfg["col_groups"] in (1, 2, 4) and cfg["item_blocks"] in (8, 16, 32)
        bk, bi, _ = oracle.knn_brute(ds, q, 8)
        np.testing.assert_array_equal(ids, bi)
        np.testing.assert_array_equal(kth, bk)
        kth2 = idx.knn(q[:100], 8, form=gts.FORM_FAST)   # small batch: the tuned config, no retuning
        np.testing.assert_array_equal(kth2, bk[:100])
        idx.fast_autotune_reset()
        assert not idx.fast_config(8)["tuned"]


def test_graph_replay_equals_direct_launches(oracle):
    """The filter pass captured in a CUDA graph and replayed gives the same
    answers as the directly launched kernels, across repeated calls and a
    change of batch shape (which captures again)."""
    rows = G.gmm_rows(25000, 128, 20, 0.2, seed=51)
    ds = oracle.Dataset(2, rows)
    q1 = G.query_ids(25000, 700, seed=52)
    q2 = G.query_ids(25000, 333, seed=53)
    with gts.Index(rows, 2, max_h=5) as idx:
        idx.fast_graphs(False)
        direct = [idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True) for q in (q1, q2)]
        idx.fast_graphs(True)
        n0 = idx.fast_graphs()
        for q, want in ((q1, direct[0]), (q1, direct[0]), (q2, direct[1]), (q2, direct[1]), (q1, direct[0])):
            got = idx.knn(q, 8, form=gts.FORM_FAST, return_ids=True)   # captured, replayed, captured, ...
            for x, y in zip(got, want):
                np.testing.assert_array_equal(x, y)
        assert idx.fast_graphs() - n0 == 5
    bk, bi, _ = oracle.knn_brute(ds, q1, 8)
    np.testing.assert_array_equal(direct[0][1], bi)


def test_fast_exact_ties_from_duplicate_rows(oracle):
    """Every row present twice: each query's candidates come in equal-distance
    pairs, so the recheck cannot certify the exact-square sums and evaluates
    the reference's pow terms; ties are broken by id."""
    base = G.gmm_rows(4000, 64, 10, 0.3, seed=61)
    rows = np.concatenate([base, base])
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(len(rows), 300, seed=62)
    with gts.Index(rows, 2, max_h=4) as idx:
        for k in (2, 7, 16):
            kth, ids, dis = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k}")


@pytest.mark.parametrize("n,dim,comps,sigma,max_h", [(20000, 128, 32, 0.2, 5), (7777, 100, 8, 0.25, 4),
                                                     (6000, 300, 16, 0.3, 4)])
def test_fast_range_counts_equal_brute_force(oracle, n, dim, comps, sigma, max_h):
    """Range counts through the tensor-core filter equal exact brute force in
    the reference's range arithmetic and the plain traversal's counts, from
    radius 0 (the query itself) to radii holding thousands of objects."""
    rows = G.gmm_rows(n, dim, comps, sigma, seed=n + 7)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(n, 300, seed=n + 8)
    with gts.Index(rows, 2, max_h=max_h) as idx:
        for frac in (0.0, 0.001, 0.01, 0.2):
            r = 0.0 if frac == 0 else float(np.float32(G.quantile_radius(2, frac, 20000, n + 9, rows=rows)))
            fast = idx.range(q, r, form=gts.FORM_FAST)
            np.testing.assert_array_equal(fast, oracle.range_brute(ds, q, r), err_msg=f"r={r}")
            np.testing.assert_array_equal(fast, idx.range(q, r), err_msg=f"r={r}")


def test_fast_range_overflow_goes_to_the_plain_traversal(oracle):
    """1,500 copies of one row just inside the radius (1e-6 relative, well
    beyond rounding, well inside the filter's 3e-5 band): every copy is
    uncertain to the filter, the query's list overflows and the plain
    traversal counts it."""
    base = G.gmm_rows(5000, 64, 8, 0.3, seed=71)
    rows = np.concatenate([base, np.repeat(base[7:8], 1500, axis=0)])
    ds = oracle.Dataset(2, rows)
    q = np.array([3, 11, 4000], np.int32)
    r = float(np.float32(oracle.dist(ds, 7, 3, False) * (1 + 1e-6)))
    with gts.Index(rows, 2, max_h=4) as idx:
        got = idx.range(q, r, form=gts.FORM_FAST)
    np.testing.assert_array_equal(got, oracle.range_brute(ds, q, r))
    assert got[0] >= 1501


def test_fast_range_extremes_and_device_entry(oracle):
    """A radius beyond every distance counts every object (all of them
    certainly inside), a tiny one only the query itself; the device-buffer
    entry point gives the host one's counts."""
    import torch
    rows = G.gmm_rows(6000, 32, 6, 0.5, seed=81)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(6000, 200, seed=82)
    with gts.Index(rows, 2, max_h=4) as idx:
        np.testing.assert_array_equal(idx.range(q, 1e6, form=gts.FORM_FAST), np.full(len(q), 6000, np.int32))
        tiny = idx.range(q, 1e-6, form=gts.FORM_FAST)
        np.testing.assert_array_equal(tiny, oracle.range_brute(ds, q, 1e-6))
        r = float(np.float32(G.quantile_radius(2, 0.02, 20000, 83, rows=rows)))
        host = idx.range(q, r, form=gts.FORM_FAST)
        d_q = torch.from_numpy(q).cuda()
        d_c = torch.empty(len(q), dtype=torch.int32, device="cuda")
        idx.range_device(d_q.data_ptr(), len(q), r, d_c.data_ptr(), form=gts.FORM_FAST)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_c.cpu().numpy(), host)
        np.testing.assert_array_equal(host, oracle.range_brute(ds, q, r))


def test_streamed_records_at_resident_widths_equal_brute_force(oracle):
    """The streamed filter (records in 64-wide K chunks through their own
    stages) pinned at widths where the resident form also fits gives the
    same exact answers, for every column-group count that fits."""
    rows = G.gmm_rows(15000, 128, 24, 0.25, seed=101)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(15000, 400, seed=102)
    with gts.Index(rows, 2, max_h=5) as idx:
        for k, cg in ((1, 4), (8, 4), (8, 1), (16, 2), (33, 2), (64, 1)):
            idx.set_fast_config(k, False, cg, 8, streamed=True)
            assert idx.fast_config(k)["streamed"]
            kth, ids, dis = idx.knn(q, k, form=gts.FORM_FAST, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k} cg={cg}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k} cg={cg}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k} cg={cg}")


def test_graphs_of_alternating_batch_shapes(oracle):
    """Batches of a few shapes in turn (one per k, as a mixed-k step runs
    them) each replay their own captured graph and keep their answers."""
    rows = G.gmm_rows(25000, 64, 20, 0.25, seed=121)
    ds = oracle.Dataset(2, rows)
    batches = [(G.query_ids(25000, 400, seed=122), 8), (G.query_ids(25000, 300, seed=123), 16),
               (G.query_ids(25000, 200, seed=124), 33)]
    with gts.Index(rows, 2, max_h=5) as idx:
        want = [oracle.knn_brute(ds, q, k)[0] for q, k in batches]
        n0 = idx.fast_graphs()
        for _ in range(3):
            for (q, k), w in zip(batches, want):
                np.testing.assert_array_equal(idx.knn(q, k, form=gts.FORM_FAST), w, err_msg=f"k={k}")
        assert idx.fast_graphs() - n0 == 9


def test_graphs_of_one_shape_with_moving_buffers(oracle):
    """Device-buffer calls of one batch shape with new output buffers each
    time: the first four buffer sets are captured and replayed, further ones
    launch directly; every answer is the same."""
    import torch
    rows = G.gmm_rows(20000, 64, 16, 0.25, seed=131)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(20000, 300, seed=132)
    want = oracle.knn_brute(ds, q, 8)[0]
    with gts.Index(rows, 2, max_h=5) as idx:
        d_q = torch.from_numpy(q).cuda()
        outs = [torch.empty(len(q), dtype=torch.float32, device="cuda") for _ in range(6)]
        n0 = idx.fast_graphs()
        for rep in range(2):
            for out in outs:
                idx.knn_device(d_q.data_ptr(), len(q), 8, out.data_ptr(), form=gts.FORM_FAST)
                torch.cuda.synchronize()
                np.testing.assert_array_equal(out.cpu().numpy(), want)
        # four captures replayed twice each; the other two buffer sets direct
        assert idx.fast_graphs() - n0 == 8


@pytest.mark.parametrize("n,dim,comps,sigma,max_h", [(20000, 128, 32, 0.2, 5), (6000, 300, 16, 0.3, 4),
                                                      (3000, 40, 3, 1.0, 4), (50, 16, 1, 1.0, 3)])
def test_seed_table_bounds_the_kth_distance(oracle, n, dim, comps, sigma, max_h):
    """The starting bounds made with the records (k-th distance over the own
    block and the nearest blocks) never fall below the exact squared k-th
    distance of the next power of two, and sit near it on mixture data."""
    rows = G.gmm_rows(n, dim, comps, sigma, seed=n + 3)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(n, min(n, 400), seed=n + 4)
    with gts.Index(rows, 2, max_h=max_h) as idx:
        assert idx.prepare(gts.FORM_FAST)
        for k in (1, 2, 7, 8, 33, 64):
            kp2 = 1 << (k - 1).bit_length()
            seeds = idx.fast_seeds(q, k).astype(np.float64)
            if kp2 > n:
                assert np.all(seeds == np.float32(np.finfo(np.float32).max)), f"k={k}"
                continue
            exact = oracle.knn_brute(ds, q, kp2)[0].astype(np.float64)
            assert np.all(seeds >= exact * exact), f"k={k}: a seed below the exact k-th distance"
            if n >= 3000:
                ratio = seeds / np.maximum(exact * exact, 1e-30)
                assert np.median(ratio) < 1.5, f"k={k}: seeds far above the k-th distance ({np.median(ratio)})"
