"""Host-side helpers of bench.py (no GPU): the workloads' batches, the
configuration record of each workload, the comparison with the reference's
saved answers, and the multi-rank launch path (`--gpus 2`, gloo ranks)."""
import json
import os
import subprocess
import sys

import numpy as np

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _args(*argv):
    return bench.parse_args(list(argv))


def test_single_k_is_one_batch():
    groups = bench.k_groups(_args(), 1000)
    assert len(groups) == 1 and groups[0][0] == 8
    np.testing.assert_array_equal(groups[0][1], np.arange(1000))


def test_mixed_k_covers_every_query_once_and_is_seeded():
    a = _args("--k-mix")
    w = bench.spec(a)
    batches = bench.make_batches(a, w, None, 10_000)
    assert [p for _, p, _ in batches] == [1, 8, 32, 64]
    allq = np.sort(np.concatenate([sel for _, _, sel in batches]))
    np.testing.assert_array_equal(allq, np.arange(10_000))
    for _, _, sel in batches:                    # roughly uniform over the four k
        assert 2000 < len(sel) < 3000
    again = bench.make_batches(a, w, None, 10_000)
    for (_, k1, s1), (_, k2, s2) in zip(batches, again):
        assert k1 == k2 and np.array_equal(s1, s2)


def test_config_names_the_workload():
    assert bench.config_dict(_args(), 1)["workload"] == "gmm1000k_d128_l2_knn"
    assert bench.config_dict(_args("--k-mix"), 1)["workload"] == "gmm1000k_d128_l2_knn_kmix"
    a = _args("--op", "range")
    a.radius = 3.0
    c = bench.config_dict(a, 1)
    assert c["workload"] == "gmm1000k_d128_l2_range" and c["radius"] == 3.0
    assert bench.config_dict(_args("--workload", "cfg0"), 1)["workload"] == "gmm50k_d300_l2_knn_range"
    assert bench.config_dict(_args("--workload", "cfg1"), 1)["workload"] == "words1000k_edit_knn_range"
    assert bench.config_dict(_args("--workload", "cfg3"), 1)["workload"] == "hotspots10000k_d2_l1_range"


def test_workload_batches_follow_the_configurations():
    w = bench.spec(_args("--workload", "cfg1"))
    b = bench.make_batches(_args("--workload", "cfg1"), w, None, 10)
    assert [(op, p) for op, p, _ in b] == [("range", 1.0), ("range", 2.0), ("range", 3.0), ("knn", 16)]
    # the quantile radius is resolved from seeded pair distances of the data
    a = _args("--workload", "cfg0", "--n", "3000")
    w = bench.spec(a)
    rows, _ = bench.make_data(w, a.seed)
    assert rows.shape == (3000, 300)
    b = bench.make_batches(a, w, rows, 5)
    assert b[0][:2] == ("knn", 8) and b[1][0] == "range" and 0 < b[1][1] < 100
    assert bench.needs_flush(w) and not bench.needs_flush(bench.spec(_args()))


def test_reference_answers_are_compared(tmp_path, monkeypatch):
    monkeypatch.setattr(bench.tempfile, "gettempdir", lambda: str(tmp_path))
    a = _args("--workload", "cfg1", "--queries", "6")
    w = bench.spec(a)
    batches = [("range", 1.0, np.arange(6)), ("knn", 16, np.arange(6))]
    got = [np.array([1, 2, 3, 4, 5, 6], np.int32), np.array([1, 1, 2, 2, 3, 3], np.float32)]
    assert bench.compare_with_reference(a, w, batches, got)["checked"] == 0
    np.savez(bench.ref_result_path(a, w), pos0=np.arange(4), val0=got[0][:4],
             pos1=np.array([5, 1, 2, 0]), val1=np.array([3, 1, 2, 1], np.float32))
    r = bench.compare_with_reference(a, w, batches, got)
    assert r["checked"] == 8 and r["agrees"] and r["identical"] == 8
    # a k-th distance off by more than the sort-code quantum disagrees
    np.savez(bench.ref_result_path(a, w), pos1=np.array([5]), val1=np.array([3.001], np.float32))
    assert not bench.compare_with_reference(a, w, batches, got)["agrees"]
    np.savez(bench.ref_result_path(a, w), pos0=np.arange(4), val0=got[0][:4] + 1)
    assert not bench.compare_with_reference(a, w, batches, got)["agrees"]
    # the quantum: one double ulp of the largest code, times INFI_DIS, times 2
    assert 3e-5 < bench.kth_quantum(100_000) < 4e-5
    assert 2e-6 < bench.kth_quantum(10_000) < 3e-6


def test_gpus_flag_launches_that_many_ranks():
    """`bench.py --gpus 2` relaunches itself under torchrun; the two ranks
    meet (gloo in the dry run) and rank 0 prints the max over ranks."""
    env = dict(os.environ, PYTHONPATH=ROOT)
    env.pop("WORLD_SIZE", None)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run",
                        "--warmup", "3"], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2 and lines[0]["max_over_ranks"] == 2.0
