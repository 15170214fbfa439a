"""The stream update's host pass (gts_update_plan) on CPU.

gts_update_run answers every query of a stream in one batched search over
the index as built, from the time intervals this pass gives each entry
(the data rows and every inserted copy).  Counting, for each query, the
entries live at its operation by brute force over the reference's F32 leaf
arithmetic (the oracle's distance) must give the oracle's answers for the
whole stream (update.cuh:449-638 restated, exact mode); the rows left after
the last compaction must be the data the oracle's restatement holds then.
"""
import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G


def _counts_from_plan(O, ds, plan, r):
    ent_src, life = plan["ent_src"], plan["ent_life"]
    out, rnum = [], 0
    cache_dist = {}
    for qo, t, has_cache in zip(plan["q_obj"], plan["q_time"], plan["q_cache"]):
        if qo not in cache_dist:
            cache_dist[qo] = np.array([O.dist(ds, int(qo), b, False) for b in range(ds.num)], np.float32)
        within = cache_dist[qo][ent_src] <= np.float32(r)
        tree = (life[:, 0] < t) & (t < life[:, 1])
        cache = (life[:, 2] < t) & (t < life[:, 3])
        if has_cache:
            rnum = int((within & cache).sum())
        out.append(int((within & tree).sum()) + rnum)
    return np.array(out, np.int32)


@pytest.mark.parametrize("max_in", [3, 10])
def test_plan_counts_equal_the_oracle_stream(oracle, max_in):
    rows = G.gmm_rows(240, 6, 5, 0.4, seed=5)
    ds = oracle.Dataset(2, rows)
    flags, ids = G.update_stream(240, 900, seed=6, max_in_size=max_in)
    r = float(np.float32(G.quantile_radius(2, 0.05, 20000, 7, rows=rows)))
    plan = gts.update_plan(240, flags, ids, max_in)
    assert len(plan["q_obj"]) == int((flags == 2).sum())
    assert len(plan["ent_src"]) == 240 + int((flags == 0).sum())
    want = oracle.update_run(ds, oracle.params(max_h=3), max_in, flags, ids, r, exact=True)
    np.testing.assert_array_equal(_counts_from_plan(oracle, ds, plan, r), want)
    # every entry copies a row of the data; the compactions happened
    assert plan["ent_src"].min() >= 0 and plan["ent_src"].max() < 240
    assert len(plan["final_rows"]) > 0


def test_plan_rows_after_the_last_compaction():
    """The final data: live rows in physical order, then the cached copies,
    compacted at every max_in-th insert (a hand-checked stream)."""
    # 5 rows; delete logical 1 (row 1), insert a copy of physical 4, insert a
    # copy of physical 0 (cache full at 2: compaction -> rows 0,2,3,4,4,0),
    # delete logical 0 (row 0, after the compaction: not applied to the data)
    flags = np.array([1, 0, 0, 1, 2], np.int32)
    ids = np.array([1, 4, 0, 0, 5], np.int32)
    plan = gts.update_plan(5, flags, ids, 2)
    np.testing.assert_array_equal(plan["final_rows"], [0, 2, 3, 4, 4, 0])
    # the query names physical row 5 of the compacted array: a copy of row 0
    assert plan["q_obj"].tolist() == [0] and plan["q_time"].tolist() == [4]
    assert plan["q_cache"].tolist() == [False]
    life = plan["ent_life"]
    assert life[1].tolist()[:2] == [-1, 0]           # row 1: deleted at op 0
    assert life[5].tolist() == [2, 2**31 - 1, 1, 2]  # copy of row 4: cached 1..2, then tree
    assert life[0].tolist()[:2] == [-1, 3]           # row 0 deleted at op 3


def test_plan_rejects_bad_ids():
    with pytest.raises(gts.GtsError):
        gts.update_plan(5, np.array([0], np.int32), np.array([9], np.int32), 10)
    with pytest.raises(gts.GtsError):
        gts.update_plan(5, np.array([2], np.int32), np.array([-1], np.int32), 10)
    with pytest.raises(gts.GtsError):
        gts.update_plan(5, np.array([3], np.int32), np.array([0], np.int32), 10)


def test_plan_with_new_rows_equals_the_oracle(oracle):
    """Inserts that bring new rows: the entries of the host pass, counted by
    brute force over the data rows followed by the new rows, give the
    oracle's counts of the same stream."""
    rows = G.gmm_rows(240, 6, 5, 0.4, seed=8)
    flags, ids = G.update_stream_new_rows(240, 900, seed=9, max_in_size=7)
    n_new = int((flags == 0).sum())
    new_rows = G.gmm_rows(n_new, 6, 5, 0.4, seed=10)
    r = float(np.float32(G.quantile_radius(2, 0.05, 20000, 11, rows=rows)))
    plan = gts.update_plan(240, flags, ids, 7, n_new=n_new)
    assert plan["ent_src"][240:].tolist() == list(range(240, 240 + n_new))
    both = oracle.Dataset(2, np.concatenate([rows, new_rows]))
    want = oracle.update_run_rows(oracle.Dataset(2, rows), 7, flags, ids, new_rows, r)
    np.testing.assert_array_equal(_counts_from_plan(oracle, both, plan, r), want)
    # the final data holds data rows and new rows
    assert plan["final_rows"].max() >= 240
