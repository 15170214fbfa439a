"""The CPU oracle: restated reference algorithm vs exact brute force, and the
oracle pinned against the reference's own outputs (golden fixtures)."""
import os

import numpy as np
import pytest

from gts_b200 import datagen as G
from tests import golden_io as GI


def _ds(O, c, data):
    if c["metric"] == 6:
        return O.Dataset(6, strs=data[0], lens=data[1])
    return O.Dataset(c["metric"], data)


@pytest.mark.parametrize("metric", [0, 1, 2, 5])
def test_restated_search_equals_brute_force(oracle, metric):
    rows = G.gmm_rows(3000, 12, 10, 0.4, seed=metric + 1)
    if metric == 5:
        rows = rows + 0.5   # keep angles away from the antipodal wrap
    ds = oracle.Dataset(metric, rows)
    p = oracle.params(max_h=4)   # 3000 -> 300 -> 30 -> 3: a perfect tree
    t = oracle.Tree(ds, p)
    assert t.tree_h == 4
    q = G.query_ids(3000, 60, 5)
    for k in (2, 8):
        v2 = oracle.knn_v2(ds, p, t, q, k)
        bf, _, _ = oracle.knn_brute(ds, q, k)
        np.testing.assert_array_equal(v2, bf)
    r = G.quantile_radius(metric, 0.005, 50000, 9, rows=rows)
    np.testing.assert_array_equal(oracle.range_v2(ds, p, t, q, r), oracle.range_brute(ds, q, r))


def test_edit_distance_restated(oracle):
    strs, lens = G.word_strings(2000, 3)
    ds = oracle.Dataset(6, strs=strs, lens=lens)
    p = oracle.params(max_h=4)
    t = oracle.Tree(ds, p)
    q = G.query_ids(2000, 40, 4)
    for r in (1.0, 2.0):
        np.testing.assert_array_equal(oracle.range_v2(ds, p, t, q, r), oracle.range_brute(ds, q, r))
    # the DP against a direct Python Levenshtein on a few pairs
    for a, b in [(0, 1), (5, 9), (17, 3)]:
        want = G._levenshtein(bytes(strs[a, :lens[a]]), bytes(strs[b, :lens[b]]))
        assert oracle.dist(ds, a, b, True) == want


def test_brute_force_ties_by_id(oracle):
    rows = np.zeros((6, 2), np.float32)
    rows[:, 0] = [0, 1, 1, 1, 2, 3]
    ds = oracle.Dataset(2, rows)
    kth, ids, dis = oracle.knn_brute(ds, [0], 3)
    assert ids.tolist() == [[0, 1, 2]]
    assert dis.tolist() == [[0.0, 1.0, 1.0]]
    assert kth[0] == 1.0


def test_brute_force_fewer_than_k(oracle):
    rows = np.arange(8, dtype=np.float32).reshape(4, 2)
    ds = oracle.Dataset(2, rows)
    kth, ids, dis = oracle.knn_brute(ds, [1], 6, infi_dis=10000)
    assert kth[0] == 10000.0
    assert ids[0, 4] == -1 and dis[0, 5] == 10000.0


def test_update_restated_simple(oracle):
    rows = G.gmm_rows(1000, 8, 4, 0.3, seed=2)
    ds = oracle.Dataset(2, rows)
    p = oracle.params(max_h=3)
    flags, ids = G.update_stream(1000, 120, seed=3, max_in_size=10)
    r = G.quantile_radius(2, 0.01, 20000, 4, rows=rows)
    counts = oracle.update_run(ds, p, 10, flags, ids, r)
    assert len(counts) == int((flags == 2).sum())
    assert (counts >= 1).all()   # queries name live rows: the object itself is a hit


def test_update_stream_ids_valid():
    flags, ids = G.update_stream(500, 2000, seed=1, max_in_size=7)
    assert set(np.unique(flags)) <= {0, 1, 2}
    assert (ids >= 0).all()


# ------------------------------------------------------------- golden pins

@pytest.mark.parametrize("name", GI.cases())
def test_oracle_tree_equals_reference_tree(oracle, name):
    c, data, qids, radii, fx = GI.load_case(name)
    if c.get("update_ops"):
        pytest.skip("the update case's tree is rebuilt during the stream")
    ds = _ds(oracle, c, data)
    p = oracle.params(max_h=c["max_h"])
    t = oracle.Tree(ds, p)
    assert t.tree_h == int(fx["tree_tree_h"])
    assert t.start_idx == int(fx["tree_start_idx"])
    np.testing.assert_array_equal(t.id_list, fx["tree_id_list"])
    ex = fx["tree_exists"].astype(bool)
    np.testing.assert_array_equal(t.exists.astype(bool), ex)
    for key in ("pid", "size", "lid", "is_leaf"):
        np.testing.assert_array_equal(getattr(t, key)[ex], fx["tree_" + key][ex], err_msg=key)
    np.testing.assert_array_equal(t.min_dis[ex], fx["tree_min_dis"][ex])


@pytest.mark.parametrize("name", GI.cases())
def test_oracle_results_equal_reference(oracle, name):
    c, data, qids, radii, fx = GI.load_case(name)
    ds = _ds(oracle, c, data)
    p = oracle.params(max_h=c["max_h"])
    if c.get("update_ops"):
        counts = oracle.update_run(ds, p, c["max_in_size"], fx["update_flags"], fx["update_ids"],
                                   float(radii[0]))
        np.testing.assert_array_equal(counts, fx["update_counts"])
        return
    t = oracle.Tree(ds, p)
    for k in c["ks"]:
        ref = fx[f"knn_k{k}"]
        v2 = oracle.knn_v2(ds, p, t, qids, k)
        np.testing.assert_array_equal(v2, ref, err_msg=f"knn k={k}")
        bf, _, _ = oracle.knn_brute(ds, qids, k)
        # the reference's quantised sort code can only swap near-ties
        np.testing.assert_allclose(bf, ref, rtol=1e-5, atol=2e-6)
    for i, r in enumerate(radii):
        ref = fx[f"range_r{i}"]
        np.testing.assert_array_equal(oracle.range_v2(ds, p, t, qids, r), ref, err_msg=f"r={r}")
        np.testing.assert_array_equal(oracle.range_brute(ds, qids, r), ref)


def _sample_or_skip():
    d = GI.sample_dir()
    if d is None or not os.path.exists(os.path.join(GI.GOLDEN, "sample_knn_k8.txt")):
        pytest.skip("reference sample data or its golden results not present")
    return d


def test_oracle_on_reference_sample(oracle):
    d = _sample_or_skip()
    metric, rows = G.read_text_rows(os.path.join(d, "sbw_example.txt"))
    qids = np.loadtxt(os.path.join(d, "sbw_example_qid.txt"), dtype=np.int32, skiprows=1)
    ds = oracle.Dataset(metric, rows)
    p = oracle.params(max_h=3)
    t = oracle.Tree(ds, p)
    for k in (8, 20):
        _, vals, _ = GI.parse_result_file(os.path.join(GI.GOLDEN, f"sample_knn_k{k}.txt"))
        ref = np.array([float(v) for v in vals], np.float32)
        got = oracle.knn_v2(ds, p, t, qids, k)
        # the reference prints "%f": compare at that resolution; angle values go
        # through acos, whose last-ulp rounding differs between libraries
        np.testing.assert_allclose(got, ref, atol=2e-6 + 1e-6)
    _, vals, _ = GI.parse_result_file(os.path.join(GI.GOLDEN, "sample_range_r30.txt"))
    ref = np.array([int(v) for v in vals])
    got = oracle.range_v2(ds, p, t, qids, 30.0)
    assert (got != ref).sum() <= 2   # only objects within an ulp of 30 degrees may differ


def test_radius_network_oracle_gradient_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(3)
    P = rng.standard_normal(M.N_PARAMS) * 0.1
    X = rng.random((40, M.N_IN))
    norm = np.concatenate([X.mean(0), X.std(0) + 0.1])
    t = rng.standard_normal(40)
    _, g = M.loss_and_grad(X, t, P, norm)
    eps = 1e-6
    for i in [0, 777, 4300, 5000, 20900, M.N_PARAMS - 1]:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        fd = (M.loss_and_grad(X, t, Pp, norm)[0] - M.loss_and_grad(X, t, Pm, norm)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])
