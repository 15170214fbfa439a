"""The multi-GPU host logic on CPU: two gloo ranks.

* query-sharded replicas: distinct query streams per rank, job time = the
  slowest rank's (all-reduce MAX);
* object-sharded search: every rank's k nearest within its shard, one
  all-gather and a (distance, id) merge equal the exact answer over all
  objects (here the oracle's brute force stands in for each rank's GPU
  search; tests/test_gpu_sharded.py runs the GPU one).
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gts_b200 import datagen as G
from gts_b200 import replicas as R


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        # replicas: the job time is the slowest rank's
        t = R.max_over_ranks(1.0 + rank, dist)
        q_seed = R.rank_query_seed(7, rank)
        # object shards over 3000 x 8 L2 rows
        rows = G.gmm_rows(3000, 8, 6, 0.4, seed=3)
        qids = G.query_ids(3000, 64, seed=4)
        lo, hi = R.shard_bounds(len(rows), world, rank)
        qrows = rows[qids]

        def local_search(qr, k):
            # the shard's k nearest for query rows that need not be in it:
            # append the query rows to the shard and search k + len(q) deep
            # (the appended rows take at most len(q) places), then keep the
            # shard's own objects
            q = qr
            ds = O.Dataset(2, np.concatenate([rows[lo:hi], qr]))
            qq = np.arange(hi - lo, hi - lo + len(q), dtype=np.int32)
            _, ids, dd = O.knn_brute(ds, qq, k + len(q))
            out_i = np.full((len(q), k), -1, np.int32)
            out_d = np.full((len(q), k), 10000.0, np.float32)
            for r in range(len(q)):
                keep = [(d, i) for d, i in zip(dd[r], ids[r]) if 0 <= i < hi - lo]
                keep = keep[:k]
                for j, (d, i) in enumerate(keep):
                    out_i[r, j] = i + lo
                    out_d[r, j] = d
            return out_i, out_d

        kth, ids, dd = R.sharded_knn(local_search, qrows, 5, 10000.0, dist)
        results[rank] = (t, q_seed, kth, ids)
    finally:
        dist.destroy_process_group()


def test_two_ranks_replicas_and_object_shards(oracle):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_worker, args=(world, port, results), nprocs=world, join=True, start_method="spawn")
        res = dict(results)
    assert res[0][0] == res[1][0] == 2.0                    # max over ranks
    assert res[0][1] != res[1][1]                           # distinct query streams
    rows = G.gmm_rows(3000, 8, 6, 0.4, seed=3)
    qids = G.query_ids(3000, 64, seed=4)
    bk, bi, _ = oracle.knn_brute(oracle.Dataset(2, rows), qids, 5)
    for r in range(world):                                   # every rank holds the global answer
        np.testing.assert_array_equal(res[r][3], bi)
        np.testing.assert_array_equal(res[r][2], bk)


def test_merge_topk_ties_and_short_shards():
    d = np.array([[[1.0, 2.0, 10000.0]], [[1.0, 1.5, 3.0]]], np.float32)
    i = np.array([[[7, 3, -1]], [[5, 9, 2]]], np.int32)
    kth, ids, dd = R.merge_topk(d, i, 3, 10000.0)
    np.testing.assert_array_equal(ids[0], [5, 7, 9])        # equal distances: smaller id first
    np.testing.assert_array_equal(dd[0], [1.0, 1.0, 1.5])
    assert kth[0] == 1.5
    kth, ids, dd = R.merge_topk(d[:1], i[:1], 3, 10000.0)   # fewer than k objects
    assert kth[0] == 10000.0 and ids[0, 2] == -1


def test_shard_bounds_cover_every_object():
    for num in (1, 7, 1000):
        for world in (1, 2, 3, 8):
            spans = [R.shard_bounds(num, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == num
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
