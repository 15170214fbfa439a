"""Host-side helpers of bench.py (no GPU): the per-k batches of the mixed-k
workload and the configuration record of each workload."""
import argparse

import numpy as np

import bench


def _args(**kw):
    a = argparse.Namespace(k=8, k_mix=False, seed=2024, n=1_000_000, dim=128, queries=10_000, max_h=6,
                           form="fast", no_learn=False, learned_seed="auto", op="knn", range_quantile=0.001)
    for key, v in kw.items():
        setattr(a, key, v)
    return a


def test_single_k_is_one_batch():
    groups = bench.k_groups(_args(), 1000)
    assert len(groups) == 1 and groups[0][0] == 8
    np.testing.assert_array_equal(groups[0][1], np.arange(1000))


def test_mixed_k_covers_every_query_once_and_is_seeded():
    a = _args(k_mix=True)
    groups = bench.k_groups(a, 10_000)
    assert [k for k, _ in groups] == [1, 8, 32, 64]
    allq = np.sort(np.concatenate([sel for _, sel in groups]))
    np.testing.assert_array_equal(allq, np.arange(10_000))
    for _, sel in groups:                       # roughly uniform over the four k
        assert 2000 < len(sel) < 3000
    again = bench.k_groups(a, 10_000)
    for (k1, s1), (k2, s2) in zip(groups, again):
        assert k1 == k2 and np.array_equal(s1, s2)


def test_config_names_the_workload():
    assert bench.config_dict(_args(), 1)["workload"] == "gmm1000k_d128_l2_knn"
    assert bench.config_dict(_args(k_mix=True), 1)["workload"] == "gmm1000k_d128_l2_knn_kmix"
    c = bench.config_dict(_args(op="range", radius=3.0), 1)
    assert c["workload"] == "gmm1000k_d128_l2_range" and c["radius"] == 3.0
