"""Multi-GPU plumbing for the GTS search path (one process per GPU).

The reference has no multi-GPU code: its queries are independent, so the
natural scale-out is query-sharded replicas (every rank holds the whole
index and answers its own queries; no collective on the data path).  For an
index larger than one GPU the objects are split into shards instead; every
rank searches its shard for all queries and one all-gather of the per-shard
top-k (k distances and ids per query) plus a per-query k-way merge by
(distance, id) gives the global answer -- the same order the reference's
ids would have (ties broken by id).

The process group is torch.distributed: NCCL over NVLink on the GPUs,
gloo for the CPU tests.  Nothing here computes distances.
"""
from __future__ import annotations

import numpy as np


def rank_query_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s query stream: distinct per rank (weak scaling)."""
    return seed + 1 + 7919 * rank


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over all ranks (the job's time is its slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_bounds(num: int, world: int, rank: int) -> tuple[int, int]:
    """Object-id range [lo, hi) of `rank`'s shard: contiguous, sizes differing
    by at most one."""
    base, extra = divmod(num, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def merge_topk(dists: np.ndarray, ids: np.ndarray, k: int, infi: float):
    """Per-query k-way merge of shard results.

    dists, ids: (shards, queries, k) -- each shard's k nearest, ascending by
    (distance, id), global ids (-1 / infi where a shard had fewer than k).
    Returns (kth, ids, dists) of the k nearest over all shards ordered by
    (distance, id); kth = infi when fewer than k objects exist."""
    s, q, kk = dists.shape
    d = np.transpose(dists, (1, 0, 2)).reshape(q, s * kk).astype(np.float64)
    i = np.transpose(ids, (1, 0, 2)).reshape(q, s * kk).astype(np.int64)
    d = np.where(i < 0, np.inf, d)
    key_id = np.where(i < 0, np.iinfo(np.int64).max, i)
    order = np.lexsort((key_id, d), axis=1)[:, :k]
    od = np.take_along_axis(d, order, axis=1)
    oi = np.take_along_axis(i, order, axis=1)
    have = np.isfinite(od)
    out_d = np.where(have, od, infi).astype(np.float32)
    out_i = np.where(have, oi, -1).astype(np.int32)
    kth = out_d[:, k - 1].copy()
    return kth, out_i, out_d


def shard_search(index, lo: int):
    """The local search of a rank whose index holds objects [lo, lo + n) of
    the global set: the shard's k nearest of query rows (not ids: a query
    need not be in this shard), global ids, on the GPU (gts_knn_rows)."""
    def search(qrows, k):
        _, ids, dists = index.knn_rows(qrows, k, return_ids=True)
        return np.where(ids >= 0, ids + lo, -1).astype(np.int32), dists
    return search


def sharded_knn(local_search, queries, k: int, infi: float, dist, device=None):
    """kNN over an object set split across the ranks of `dist`.

    local_search(queries, k) -> (ids, dists): this rank's shard's k nearest
    per query (global ids, ascending by (distance, id)); queries are the
    query rows every rank holds.  One all-gather of the (queries x k)
    distances and ids, then merge_topk.  Every rank returns the global
    answer."""
    import torch
    ids, dists = local_search(queries, k)
    world = dist.get_world_size()
    td = torch.as_tensor(np.ascontiguousarray(dists, dtype=np.float32), device=device)
    ti = torch.as_tensor(np.ascontiguousarray(ids, dtype=np.int32), device=device)
    gd = [torch.empty_like(td) for _ in range(world)]
    gi = [torch.empty_like(ti) for _ in range(world)]
    dist.all_gather(gd, td)
    dist.all_gather(gi, ti)
    D = np.stack([x.cpu().numpy() for x in gd])
    I = np.stack([x.cpu().numpy() for x in gi])
    return merge_topk(D, I, k, infi)
