"""Generate golden fixtures by running the reference GTS build.

Run on a machine with a CUDA GPU after `make -C oracle ref` (the reference's
own CUDA build, compiled from the reference sources).  For every case below
it regenerates the seeded data set, runs the reference harness
(oracle/_ref/gts_ref_driver) for kNN / range / update, and stores the
reference's outputs plus the reference's built tree in tests/golden/<case>.npz.
The data itself is not stored: tests regenerate it from the recorded seeds
and check the stored checksum.

The sample data set of the reference checkout (Datasets Sample/) is run
through the reference's unmodified CLI (oracle/_ref/GTS) when --sample names
a directory holding it; its result files are stored as text.

Tree parameters are chosen so that every tree is "perfect" (every node above
the last level holds more than MAX_SIZE objects, every last-level node at most
MAX_SIZE) -- the shapes on which the reference's v2 search is exact -- and
k stays at or below MAX_SIZE except where no pruning level exists, so every
run stays inside the reference's list-table slices.

usage: python tests/golden/make_fixtures.py --ref oracle/_ref --out DIR [--sample DIR]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from gts_b200 import datagen as G  # noqa: E402

# name: dict(kind, n, dim, metric, seed, max_h, nq, ks, radii quantiles, update ops)
CASES = {
    "l2_n2000_d16": dict(kind="gmm", n=2000, dim=16, comps=16, sigma=0.3, metric=2, seed=11,
                         max_h=3, nq=200, ks=[1, 5, 20], rq=[0.001, 0.01]),
    "l2_n5000_d32": dict(kind="gmm", n=5000, dim=32, comps=32, sigma=0.3, metric=2, seed=12,
                         max_h=4, nq=200, ks=[2, 8, 20], rq=[0.001, 0.01]),
    "l2_n3333_d8": dict(kind="gmm", n=3333, dim=8, comps=8, sigma=0.5, metric=2, seed=13,
                        max_h=4, nq=150, ks=[2, 8], rq=[0.002]),
    "l1_n20000_d2": dict(kind="hot", n=20000, dim=2, metric=1, seed=14, max_h=4, nq=200,
                         ks=[2, 16], rq=[0.0005, 0.002]),
    "linf_n4000_d6": dict(kind="gmm", n=4000, dim=6, comps=12, sigma=0.4, metric=0, seed=15,
                          max_h=4, nq=150, ks=[3, 10], rq=[0.002]),
    "edit_n3000": dict(kind="words", n=3000, metric=6, seed=16, max_h=4, nq=150, ks=[2, 16],
                       radii=[1, 2, 3]),
    "upd_l2_n1000_d16": dict(kind="gmm", n=1000, dim=16, comps=8, sigma=0.3, metric=2, seed=17,
                             max_h=3, nq=0, ks=[], rq=[0.01], update_ops=300, max_in_size=10),
}


def make_case_data(c):
    """Deterministic data for a case: (rows | (strs, lens), qids, radii, update)."""
    if c["kind"] == "gmm":
        rows = G.gmm_rows(c["n"], c["dim"], c["comps"], c["sigma"], c["seed"])
    elif c["kind"] == "hot":
        rows = G.hotspot_points(c["n"], c["seed"], n_hot=50)
    else:
        rows = None
    if c["kind"] == "words":
        strs, lens = G.word_strings(c["n"], c["seed"])
        data = (strs, lens)
        digest = hashlib.sha1(strs.tobytes() + lens.tobytes()).hexdigest()
    else:
        data = rows
        digest = hashlib.sha1(rows.tobytes()).hexdigest()
    qids = G.query_ids(c["n"], c["nq"], c["seed"] + 1000) if c["nq"] else np.zeros(0, np.int32)
    if "radii" in c:
        radii = [float(r) for r in c["radii"]]
    else:
        radii = [float(np.float32(G.quantile_radius(c["metric"], q, 200000, c["seed"] + 2000,
                                                    rows=rows))) for q in c["rq"]]
    upd = None
    if c.get("update_ops"):
        upd = G.update_stream(c["n"], c["update_ops"], c["seed"] + 3000, c["max_in_size"])
    return data, digest, qids, radii, upd


def read_tree(path):
    raw = np.fromfile(path, dtype=np.int32)
    n, mnn, tree_h, start_idx = raw[:4]
    id_list = raw[4:4 + n]
    rec = raw[4 + n:4 + n + 6 * mnn].reshape(mnn, 6)
    return dict(id_list=id_list, pid=rec[:, 0], min_dis=rec[:, 1].view(np.float32),
                size=rec[:, 2], lid=rec[:, 3], is_leaf=rec[:, 4], exists=rec[:, 5],
                tree_h=int(tree_h), start_idx=int(start_idx))


def run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    last = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    return json.loads(last[-1]) if last else {}


def gen_case(name, c, driver, tmp, out):
    data, digest, qids, radii, upd = make_case_data(c)
    dpath = os.path.join(tmp, name + (".txt" if c["metric"] == 6 else ".bin"))
    if c["metric"] == 6:
        G.write_data_text(dpath, 6, strs=data[0], lens=data[1])
    else:
        G.write_data_bin(dpath, c["metric"], data)
    qpath = os.path.join(tmp, name + "_q.txt")
    G.write_queries(qpath, qids)
    common = ["--order", "10", "--max-size", "20", "--max-h", str(c["max_h"]), "--budget-gb", "6"]
    if c["metric"] == 6:
        common[-1] = "7"    # range sizes are int-typed: under 8 GB
    res = dict(case=json.dumps(c), digest=digest, qids=qids, radii=np.array(radii, np.float32))
    tree_path = os.path.join(tmp, name + ".tree")
    rpath = os.path.join(tmp, name + ".res")
    outp = os.path.join(tmp, name + ".out")
    first = True
    for k in c["ks"]:
        extra = ["--dump-tree", tree_path] if first else []
        run([driver, dpath, qpath, "0", str(k), outp, *common, *extra, "--dump-res", rpath])
        res[f"knn_k{k}"] = np.fromfile(rpath, dtype=np.float32)
        first = False
    for i, r in enumerate(radii):
        extra = ["--dump-tree", tree_path] if first else []
        if c.get("update_ops"):
            flags, ids = upd
            upath = os.path.join(tmp, name + "_u.txt")
            G.write_updates(upath, flags, ids)
            run([driver, dpath, upath, "2", repr(r), outp, *common, *extra,
                 "--max-in-size", str(c["max_in_size"])])
            with open(outp) as f:
                lines = f.read().splitlines()
            res["update_counts"] = np.array([int(v) for v in lines[2].split()], np.int32)
            res["update_flags"], res["update_ids"] = flags, ids
        else:
            run([driver, dpath, qpath, "1", repr(r), outp, *common, *extra, "--dump-res", rpath])
            res[f"range_r{i}"] = np.fromfile(rpath, dtype=np.int32)
        first = False
    t = read_tree(tree_path)
    for key, v in t.items():
        res["tree_" + key] = np.asarray(v)
    np.savez_compressed(os.path.join(out, name + ".npz"), **res)
    print(f"{name}: ok ({', '.join(k for k in res if k.startswith(('knn', 'range', 'update_c')))})")


def gen_sample(driver, sample_dir, out):
    """The reference on its own sample data (README.md:49-84), text files read
    by its own loader, default tree parameters (MAX_H 3).

    The unmodified CLI (src/main.cu) cannot run on a 180 GB B200: it sizes its
    list table as half the free memory in an int count of elements
    (search_v2.cuh:995-1001), which overflows, and stops with "out of memory".
    The harness runs the same entry points with a 6 GB list-table budget."""
    data = os.path.join(sample_dir, "sbw_example.txt")
    qid = os.path.join(sample_dir, "sbw_example_qid.txt")
    upd = os.path.join(sample_dir, "sbw_example_u.txt")
    runs = {"sample_knn_k8.txt": [data, qid, "0", "8"],
            "sample_knn_k20.txt": [data, qid, "0", "20"],
            "sample_range_r30.txt": [data, qid, "1", "30"],
            "sample_update_r59.txt": [data, upd, "2", "59"]}
    for fname, args in runs.items():
        dst = os.path.join(out, fname)
        run([driver, *args, dst, "--max-h", "3", "--budget-gb", "6"])
        print(f"{fname}: ok")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.path.join(HERE, "..", "..", "oracle", "_ref"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--sample", default=None)
    ap.add_argument("--cases", default=",".join(CASES))
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    driver = os.path.join(a.ref, "gts_ref_driver")
    tmp = tempfile.mkdtemp(prefix="gts_golden_")
    try:
        for name in [c for c in a.cases.split(",") if c and c != "none"]:
            gen_case(name, CASES[name], driver, tmp, a.out)
        if a.sample:
            gen_sample(driver, a.sample, a.out)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
