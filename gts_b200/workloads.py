"""Representative runs of every kernel family of the GTS path, scaled down
from the benchmark configurations (seeded synthetic data in the configs'
shapes and distributions), for profiling and smoke runs:

    python -m gts_b200.workloads [--scale 0.1]

* L2 (Gaussian mixture, 128-d): tree build, filter block order and records,
  learned-radius training and inference, fast kNN, plain kNN (unseeded and
  seeded by the learned radius), range counts (plain and tensor-core), range
  ids;
* edit distance (Zipf words): build, kNN and range;
* L1 (2-D hotspots): build and range;
* streaming updates (L2): inserts, deletes and range queries through the
  lazy cache list with rebuilds.

Every result is checked against another form of the same search (the fast
form against the plain traversal, seeded against unseeded) so a profiled
run is also a consistency run.
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

import gts_b200 as gts
from gts_b200 import datagen as G


def _t(label, f, *a, **kw):
    t0 = time.perf_counter()
    out = f(*a, **kw)
    print(f"  {label}: {time.perf_counter() - t0:.3f} s", flush=True)
    return out


def run(scale: float = 0.1, seed: int = 11) -> None:
    n = max(4000, int(1_000_000 * scale))
    q = max(256, int(10_000 * scale))
    print(f"L2 mixture {n} x 128, {q} queries", flush=True)
    rows = G.gmm_rows(n, 128, 256, 0.2, seed=seed)
    qids = G.query_ids(n, q, seed=seed + 1)
    with _t("build", gts.Index, rows, 2, max_h=6 if n >= 400_000 else 5) as idx:
        fast = _t("fast kNN k=8 (first call: block order, records, autotune)", idx.knn, qids, 8, form=gts.FORM_FAST)
        plain = _t("plain kNN k=8", idx.knn, qids[: max(64, q // 10)], 8, form=gts.FORM_PLAIN)
        assert np.array_equal(fast[: len(plain)], plain), "fast and plain kNN differ"
        _t("learn radius", idx.learn_radius, n_train=max(2000, q * 4), k_max=64, epochs=4, seed=seed)
        seeded = _t("plain kNN k=8 seeded by the learned radius", idx.knn, qids[: len(plain)], 8,
                    form=gts.FORM_PLAIN_LEARNED)
        assert np.array_equal(seeded, plain), "seeded and unseeded traversal differ"
        for k in (32, 64):
            _t(f"fast kNN k={k}", idx.knn, qids, k, form=gts.FORM_FAST)
        r = float(np.float32(G.quantile_radius(2, 0.001, 20000, seed + 2, rows=rows)))
        counts = _t("range counts", idx.range, qids[: len(plain)], r)
        fast_counts = _t("range counts, tensor-core filter", idx.range, qids, r, form=gts.FORM_FAST)
        assert np.array_equal(fast_counts[: len(plain)], counts), "fast and plain range counts differ"
        ids = _t("range ids", idx.range_ids, qids[: len(plain) // 4], r)
        assert np.array_equal(ids[0], counts[: len(plain) // 4]), "range ids and counts differ"
    ne = max(4000, int(1_000_000 * scale))
    print(f"edit distance, {ne} words", flush=True)
    strs, lens = G.word_strings(ne, seed=seed + 3)
    with _t("build", gts.Index, None, 6, strs=strs, lens=lens, max_h=5) as idx:
        qe = G.query_ids(ne, max(64, q // 10), seed=seed + 4)
        _t("kNN k=16", idx.knn, qe, 16)
        for rr in (1, 2, 3):
            _t(f"range r={rr}", idx.range, qe, float(rr))
    n1 = max(10_000, int(10_000_000 * scale))
    print(f"L1 hotspots {n1} x 2", flush=True)
    pts = G.hotspot_points(n1, seed=seed + 5)
    with _t("build", gts.Index, pts, 1, max_h=7 if n1 >= 2_000_000 else 6) as idx:
        q1 = G.query_ids(n1, max(256, q), seed=seed + 6)
        r1 = float(np.float32(G.quantile_radius(1, 0.0001, 20000, seed + 7, rows=pts)))
        _t("range", idx.range, q1, r1)
    nu = max(4000, int(1_000_000 * scale) // 4)
    print(f"stream updates on {nu} x 300 L2", flush=True)
    base = G.gmm_rows(nu, 300, 64, 0.3, seed=seed + 8)
    with _t("build", gts.Index, base, 2, max_h=5, max_in_size=10) as idx:
        flags, ids = G.update_stream(nu, 400, seed=seed + 9)
        ru = float(np.float32(G.quantile_radius(2, 0.001, 20000, seed + 10, rows=base)))
        _t("update stream (400 ops)", idx.update_run, flags, ids, ru)
    print("workloads ok", flush=True)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--scale", type=float, default=0.1, help="fraction of the benchmark sizes")
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    run(a.scale, a.seed)
    return 0


if __name__ == "__main__":
    sys.exit(main())
