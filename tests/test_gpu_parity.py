"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the reference's own outputs (golden fixtures).  Bit-exact for every value."""
import os

import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G
from tests import golden_io as GI

pytestmark = pytest.mark.gpu


def _ds(O, metric, data):
    if metric == 6:
        return O.Dataset(6, strs=data[0], lens=data[1])
    return O.Dataset(metric, data)


def _index(metric, data, **kw):
    if metric == 6:
        return gts.Index(None, 6, strs=data[0], lens=data[1], **kw)
    return gts.Index(data, metric, **kw)


def _data(metric, n, dim, seed):
    if metric == 6:
        return G.word_strings(n, seed)
    rows = G.gmm_rows(n, dim, max(2, n // 300), 0.4, seed)
    if metric == 5:
        rows = rows + 0.5
    return rows


SHAPES = [  # (metric, n, dim, max_h)
    (2, 3000, 16, 4), (2, 4321, 33, 4), (1, 5000, 3, 4), (0, 3000, 7, 4), (5, 2500, 24, 4),
    (6, 3000, 1, 4), (2, 2090, 8, 6),   # the last one: shallow leaves (non-perfect tree)
]


@pytest.mark.parametrize("metric,n,dim,max_h", SHAPES)
def test_tree_equals_oracle(oracle, metric, n, dim, max_h):
    data = _data(metric, n, dim, seed=n)
    p = oracle.params(max_h=max_h)
    t = oracle.Tree(_ds(oracle, metric, data), p)
    with _index(metric, data, max_h=max_h) as idx:
        e = idx.export()
    assert e["tree_h"] == t.tree_h
    if max_h == 6:
        # non-perfect tree: the reference's global sort carries stale keys of
        # finished leaves; compare the node structure, which does not depend on it
        np.testing.assert_array_equal(e["size"], t.size)
        np.testing.assert_array_equal(e["exists"], t.exists)
        return
    np.testing.assert_array_equal(e["id_list"], t.id_list)
    ex = t.exists.astype(bool)
    np.testing.assert_array_equal(e["exists"].astype(bool), ex)
    for key in ("pid", "size", "lid", "is_leaf"):
        np.testing.assert_array_equal(e[key][ex], getattr(t, key)[ex], err_msg=key)
    if metric == 5:
        # angle goes through acosf, whose last bit differs between the host
        # library and the device (the device value is the reference's)
        np.testing.assert_array_max_ulp(e["min_dis"][ex], t.min_dis[ex], maxulp=4)
    else:
        np.testing.assert_array_equal(e["min_dis"][ex], t.min_dis[ex])


@pytest.mark.parametrize("metric,n,dim,max_h", SHAPES)
def test_knn_equals_brute_force(oracle, metric, n, dim, max_h):
    data = _data(metric, n, dim, seed=n + 1)
    ds = _ds(oracle, metric, data)
    q = G.query_ids(n, 120, seed=n + 2)
    with _index(metric, data, max_h=max_h) as idx:
        for k in (1, 7, 32):
            kth, ids, dis = idx.knn(q, k, return_ids=True)
            bkth, bids, bdis = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(kth, bkth, err_msg=f"k={k}")
            np.testing.assert_array_equal(ids, bids, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bdis, err_msg=f"k={k}")


@pytest.mark.parametrize("metric,n,dim,max_h", SHAPES)
def test_range_equals_brute_force(oracle, metric, n, dim, max_h):
    data = _data(metric, n, dim, seed=n + 3)
    ds = _ds(oracle, metric, data)
    q = G.query_ids(n, 120, seed=n + 4)
    radii = [1.0, 3.0] if metric == 6 else [
        float(np.float32(G.quantile_radius(metric, f, 30000, 5, rows=data))) for f in (0.002, 0.02)]
    with _index(metric, data, max_h=max_h) as idx:
        for r in radii:
            np.testing.assert_array_equal(idx.range(q, r), oracle.range_brute(ds, q, r), err_msg=f"r={r}")


def test_range_ids(oracle):
    rows = _data(2, 4000, 12, 7)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(4000, 50, 8)
    r = float(np.float32(G.quantile_radius(2, 0.01, 30000, 9, rows=rows)))
    with gts.Index(rows, 2, max_h=4) as idx:
        counts, offs, ids, dis = idx.range_ids(q, r)
    np.testing.assert_array_equal(counts, oracle.range_brute(ds, q, r))
    for i, qid in enumerate(q):
        got = ids[offs[i]:offs[i] + counts[i]]
        assert len(set(got.tolist())) == counts[i]
        for j, o in enumerate(got):
            want = 0.0 if o == qid else oracle.dist(ds, int(o), int(qid), False)
            assert np.float32(want) <= np.float32(r)
            assert dis[offs[i] + j] == np.float32(want)


def test_plain_thread_counts_agree_and_autotuner_picks_one(oracle):
    """Every threads-per-query-CTA choice of the plain traversal gives the
    same exact answers; a large enough batch tunes the choice."""
    rows = _data(2, 12000, 24, 17)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(12000, 6000, 18)
    r = float(np.float32(G.quantile_radius(2, 0.005, 30000, 19, rows=rows)))
    bk, bi, bd = oracle.knn_brute(ds, q[:200], 8)
    bc = oracle.range_brute(ds, q[:200], r)
    with gts.Index(rows, 2, max_h=4) as idx:
        assert idx.plain_threads(0) == 0
        kth = idx.knn(q, 8)
        assert idx.plain_threads(0) in (128, 256, 512)
        counts = idx.range(q, r)
        assert idx.plain_threads(1) in (128, 256, 512)
        for nt in (128, 256, 512):
            for m in (0, 1, 2):
                idx.set_plain_threads(m, nt)
            k2, ids, dis = idx.knn(q[:200], 8, return_ids=True)
            np.testing.assert_array_equal(k2, bk)
            np.testing.assert_array_equal(ids, bi)
            np.testing.assert_array_equal(dis, bd)
            np.testing.assert_array_equal(idx.range(q[:200], r), bc)
            c2, _, _, _ = idx.range_ids(q[:200], r)
            np.testing.assert_array_equal(c2, bc)
        with pytest.raises(Exception):
            idx.set_plain_threads(0, 96)
    np.testing.assert_array_equal(kth[:200], bk)
    np.testing.assert_array_equal(counts[:200], bc)


def test_v1_entry_points(oracle, tmp_path):
    """searchIndexKnn / searchIndexRnn (the reference's v1 multi-query
    search): flat id/distance arrays, count + prefix layout, cost file."""
    rows = _data(2, 3000, 10, 23)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(3000, 40, 24)
    r = float(np.float32(G.quantile_radius(2, 0.01, 20000, 25, rows=rows)))
    bk, bi, bd = oracle.knn_brute(ds, q, 5)
    bc = oracle.range_brute(ds, q, r)
    cost = tmp_path / "cost.txt"
    with gts.indexConstru(rows, 2, max_h=4) as idx:
        ids, dis = gts.searchIndexKnn(idx, q, 5, fcost=str(cost))
        np.testing.assert_array_equal(ids, bi.reshape(-1))
        np.testing.assert_array_equal(dis, bd.reshape(-1))
        assert cost.read_text() == "".join("%f " % v for v in bk)
        cost.unlink()
        counts, prefix, rid, rdis = gts.searchIndexRnn(idx, q, r, fcost=str(cost))
    np.testing.assert_array_equal(counts, bc)
    np.testing.assert_array_equal(prefix, np.concatenate([[0], np.cumsum(bc)[:-1]]))
    assert len(rid) == len(rdis) == bc.sum()
    assert cost.read_text() == "".join("%d " % v for v in bc)


def test_update_equals_oracle(oracle):
    rows = _data(2, 1500, 10, 11)
    ds = oracle.Dataset(2, rows)
    flags, ids = G.update_stream(1500, 400, seed=12, max_in_size=10)
    r = float(np.float32(G.quantile_radius(2, 0.01, 30000, 13, rows=rows)))
    p = oracle.params(max_h=3)
    # 1500 rows drift to sizes whose last-level nodes exceed MAX_SIZE after
    # rebuilds; the reference skips those, the exact count does not
    want = oracle.update_run(ds, p, 10, flags, ids, r, exact=True)
    with gts.Index(rows, 2, max_h=3, max_in_size=10) as idx:
        got, ts, tu = idx.update_run(flags, ids, r)
    np.testing.assert_array_equal(got, want)


def test_update_with_new_rows_equals_oracle(oracle):
    """Inserts that bring new mixture samples (the stream-update
    configuration's inserts; the reference can only copy rows): the counts
    equal the oracle's exact restatement, and afterwards the handle holds
    the data of the last compaction (kNN over it equals brute force)."""
    rows = _data(2, 3000, 12, 21)
    flags, ids = G.update_stream_new_rows(3000, 1500, seed=22, max_in_size=10)
    n_new = int((flags == 0).sum())
    new_rows = G.gmm_rows(n_new, 12, 6, 0.3, seed=23)
    r = float(np.float32(G.quantile_radius(2, 0.01, 30000, 24, rows=rows)))
    want = oracle.update_run_rows(oracle.Dataset(2, rows), 10, flags, ids, new_rows, r)
    plan = gts.update_plan(3000, flags, ids, 10, n_new=n_new)
    with gts.Index(rows, 2, max_h=3, max_in_size=10) as idx:
        got, ts, tu = idx.update_run_rows(flags, ids, new_rows, r)
        np.testing.assert_array_equal(got, want)
        final = np.concatenate([rows, new_rows])[plan["final_rows"]]
        assert idx.info["num"] == len(final)
        q = np.arange(0, len(final), 37, dtype=np.int32)
        np.testing.assert_array_equal(idx.knn(q, 5), oracle.knn_brute(oracle.Dataset(2, final), q, 5)[0])


# ------------------------------------------------------------- edge cases

def test_k_larger_than_n_and_self():
    rows = G.gmm_rows(30, 4, 2, 0.5, 3)
    with gts.Index(rows, 2, max_h=2) as idx:
        kth = idx.knn([0, 5], 50)
        assert (kth == 10000.0).all()
        k1, ids, dis = idx.knn([0, 5, 29], 1, return_ids=True)
        assert k1.tolist() == [0.0, 0.0, 0.0]
        assert ids[:, 0].tolist() == [0, 5, 29]


def test_empty_query_batch_and_bad_args():
    rows = G.gmm_rows(100, 4, 2, 0.5, 3)
    with gts.Index(rows, 2, max_h=2) as idx:
        assert idx.knn(np.zeros(0, np.int32), 3).shape == (0,)
        with pytest.raises(gts.GtsError):
            idx.knn([0], 0)
        with pytest.raises(gts.GtsError):
            idx.knn([100], 3)
        with pytest.raises(gts.GtsError):
            idx.range([-1], 1.0)


def test_root_only_tree_and_duplicates(oracle):
    rows = np.tile(G.gmm_rows(5, 3, 1, 0.1, 1), (400, 1))   # 2000 rows, 5 distinct values
    ds = oracle.Dataset(2, rows)
    q = np.arange(0, 2000, 97, dtype=np.int32)
    for max_h in (1, 3):
        with gts.Index(rows, 2, max_h=max_h) as idx:
            kth, ids, dis = idx.knn(q, 9, return_ids=True)
            bk, bi, bd = oracle.knn_brute(ds, q, 9)
            np.testing.assert_array_equal(ids, bi)
            np.testing.assert_array_equal(kth, bk)
            np.testing.assert_array_equal(idx.range(q, 0.0), oracle.range_brute(ds, q, 0.0))


def test_large_leaves(oracle):
    """Nodes above max_size at the last level (is_leaf == 0) are still searched."""
    rows = G.gmm_rows(6000, 6, 5, 0.3, 21)
    ds = oracle.Dataset(2, rows)
    q = G.query_ids(6000, 40, 22)
    with gts.Index(rows, 2, max_h=2) as idx:   # 10 leaves of 600 objects
        kth, ids, _ = idx.knn(q, 16, return_ids=True)
        bk, bi, _ = oracle.knn_brute(ds, q, 16)
        np.testing.assert_array_equal(ids, bi)


# ------------------------------------------------------------- golden pins

@pytest.mark.parametrize("name", GI.cases())
def test_gpu_equals_reference_goldens(oracle, name):
    c, data, qids, radii, fx = GI.load_case(name)
    metric = c["metric"]
    with _index(metric, data, max_h=c["max_h"], max_in_size=c.get("max_in_size", 10)) as idx:
        if c.get("update_ops"):
            got, _, _ = idx.update_run(fx["update_flags"], fx["update_ids"], float(radii[0]))
            np.testing.assert_array_equal(got, fx["update_counts"])
            return
        e = idx.export()
        np.testing.assert_array_equal(e["id_list"], fx["tree_id_list"])
        ex = fx["tree_exists"].astype(bool)
        np.testing.assert_array_equal(e["min_dis"][ex], fx["tree_min_dis"][ex])
        for k in c["ks"]:
            got = idx.knn(qids, k)
            ref = fx[f"knn_k{k}"]
            # identical except where the reference's quantised sort code swapped
            # a near-tie (|difference| below its code quantum)
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-6)
            assert (got == ref).mean() > 0.98
        for i, r in enumerate(radii):
            np.testing.assert_array_equal(idx.range(qids, float(r)), fx[f"range_r{i}"])


@pytest.mark.parametrize("name", [c for c in GI.cases() if c.startswith("l2_")])
def test_fast_form_equals_reference_goldens(oracle, name):
    """The tensor-core form pinned to the reference's own outputs (not only
    through the oracle): k-th distances equal up to the reference's sort-code
    quantum, range counts exactly."""
    c, data, qids, radii, fx = GI.load_case(name)
    with _index(c["metric"], data, max_h=c["max_h"]) as idx:
        for k in c["ks"]:
            got = idx.knn(qids, k, form=gts.FORM_FAST)
            ref = fx[f"knn_k{k}"]
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-6)
            assert (got == ref).mean() > 0.98
            np.testing.assert_array_equal(got, idx.knn(qids, k))   # = the plain form, exactly
        for i, r in enumerate(radii):
            np.testing.assert_array_equal(idx.range(qids, float(r), form=gts.FORM_FAST), fx[f"range_r{i}"])


def test_gpu_on_reference_sample(oracle):
    d = GI.sample_dir()
    if d is None or not os.path.exists(os.path.join(GI.GOLDEN, "sample_knn_k8.txt")):
        pytest.skip("reference sample data or its golden results not present")
    dim, n, metric, rows = gts.load(os.path.join(d, "sbw_example.txt"))
    qids = gts.load_queries(os.path.join(d, "sbw_example_qid.txt"))
    with gts.Index(rows, metric, max_h=3) as idx:
        for k in (8, 20):
            _, vals, _ = GI.parse_result_file(os.path.join(GI.GOLDEN, f"sample_knn_k{k}.txt"))
            got = idx.knn(qids, k)
            assert [f"{v:f}" for v in got] == vals
        _, vals, _ = GI.parse_result_file(os.path.join(GI.GOLDEN, "sample_range_r30.txt"))
        assert [str(v) for v in idx.range(qids, 30.0)] == vals
    f, i = gts.load_updates(os.path.join(d, "sbw_example_u.txt"))
    with gts.Index(rows, metric, max_h=3) as idx:
        got, _, _ = idx.update_run(f, i, 59.0)
    _, vals, _ = GI.parse_result_file(os.path.join(GI.GOLDEN, "sample_update_r59.txt"))
    assert [str(v) for v in got] == vals
