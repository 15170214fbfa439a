"""The object-sharded kNN on the GPU: two ranks (gloo processes sharing the
one GPU of a test box; their kernels never wait on each other) each build
the index of their half of the objects, search it for query rows they may
not hold (gts_knn_rows), and one all-gather plus the (distance, id) merge
gives every rank the exact global answer."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gts_b200 import datagen as G
from gts_b200 import replicas as R

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import gts_b200 as gts
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = G.gmm_rows(12000, 24, 10, 0.3, seed=91)
        qids = G.query_ids(12000, 300, seed=92)
        lo, hi = R.shard_bounds(len(rows), world, rank)
        with gts.Index(rows[lo:hi], 2, max_h=3) as idx:
            kth, ids, dd = R.sharded_knn(R.shard_search(idx, lo), rows[qids], 9, 10000.0, dist)
        results[rank] = (kth, ids, dd)
    finally:
        dist.destroy_process_group()


def test_object_sharded_knn_on_the_gpu_equals_brute_force(oracle):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_worker, args=(world, port, results), nprocs=world, join=True, start_method="spawn")
        res = dict(results)
    rows = G.gmm_rows(12000, 24, 10, 0.3, seed=91)
    qids = G.query_ids(12000, 300, seed=92)
    bk, bi, bd = oracle.knn_brute(oracle.Dataset(2, rows), qids, 9)
    for r in range(world):
        np.testing.assert_array_equal(res[r][1], bi)
        np.testing.assert_array_equal(res[r][0], bk)
        np.testing.assert_array_equal(res[r][2], bd)


def test_knn_rows_equals_knn_by_id(oracle):
    """Query rows that are objects of the index give the answers of the
    same queries by id (L2: an object's distance to its own row is 0), and
    rows outside the index match brute force over an extended set."""
    import gts_b200 as gts
    rows = G.gmm_rows(8000, 40, 12, 0.3, seed=93)
    qids = G.query_ids(8000, 200, seed=94)
    extra = G.gmm_rows(50, 40, 12, 0.3, seed=95)
    with gts.Index(rows, 2, max_h=4) as idx:
        a = idx.knn(qids, 7, return_ids=True)
        b = idx.knn_rows(rows[qids], 7, return_ids=True)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
        r = float(np.float32(G.quantile_radius(2, 0.01, 20000, 96, rows=rows)))
        np.testing.assert_array_equal(idx.range_rows(rows[qids], r), idx.range(qids, r))
        kth, ids, _ = idx.knn_rows(extra, 5, return_ids=True)
    both = np.concatenate([rows, extra])
    ds = oracle.Dataset(2, both)
    # each extra row searched in (rows + extra): its own row sits at 0; drop
    # the appended rows from the brute-force lists
    _, bi, bd = oracle.knn_brute(ds, np.arange(8000, 8050, dtype=np.int32), 5 + 50)
    for j in range(50):
        keep = [(d, i) for d, i in zip(bd[j], bi[j]) if i < 8000][:5]
        np.testing.assert_array_equal(ids[j], [i for _, i in keep])
        assert kth[j] == keep[-1][0]
