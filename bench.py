"""Benchmark: exact metric-search queries/s on one B200 (GTS similarity-search path).

Workloads (--workload; seeded synthetic data stand in for the paper's data
sets, which are not available, at the same shapes and distributions):

  cfg2 (default, the headline)  1,000,000 x 128 float32 L2 rows from a
      256-component Gaussian mixture (sigma 0.2); 10,000 concurrent kNN
      queries, k = 8 (--k-mix: k uniform over {1, 8, 32, 64}, one batch per
      k; --op range: range counts at the 0.1 % distance quantile); tree
      O 10 / S 20 / MAX_H 6 (a perfect tree: 100,000 leaves of 10 objects)
  cfg0  50,000 x 300 float32 L2 rows (64-component mixture, sigma 0.3);
      1,000 kNN queries at k = 8 plus the same 1,000 as range queries at
      the 0.1 % distance quantile; MAX_H 5
  cfg1  1,000,000 lowercase strings (log-normal lengths 1..34, median 8,
      Zipf(1.1) letters), edit distance; 10,000 range queries at r = 1, 2
      and 3 plus kNN at k = 16; MAX_H 6
  cfg3  10,000,000 two-dimensional float32 points (70 % in 500 Gaussian
      hotspots of sigma 0.005, 30 % uniform), L1; 100,000 range queries at
      the 0.01 % distance quantile; MAX_H 7
  cfg4  stream update on 1,000,000 x 300 L2 rows (the cfg0 mixture at 1M):
      a seeded stream of --ops operations (45 % insert, 45 % delete, 10 %
      range query at the 0.1 % quantile) through the lazy cache list of 10
      entries, then the rebuild of the final data set

One step = every batch of the workload once (cfg4: the whole stream).
value = queries (cfg4: operations) of one step / step time, device-timed
with CUDA events.  Each workload's data set is larger than the 126 MB L2
except cfg0 (60 MB) and cfg3's 80 MB, where every step starts by writing a
256 MB buffer (L2 flush, outside the timed events).

    python bench.py [--workload cfg2] [--gpus N] [--steps K] [--warmup W]
                    [--impl gts|reference] [--form fast|plain|plain-learned]

--impl reference runs the reference's own CUDA build (oracle/_ref, built
from the reference sources) through its entry points on the same data and
prints the same JSON line with "impl": "reference"; it saves its answers so
that the next gts run on the same workload compares every answer the
reference gave (agrees_with_reference).

Multi-GPU: one rank per GPU (torchrun; `--gpus N` without torchrun relaunches
itself under it).  Every rank holds a replica of the index and answers its
own queries (weak scaling, no collective on the data path); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
BF16_FALLBACK_TFLOPS = 1590.0
K_MIX = (1, 8, 32, 64)

# The reference sizes its list table as half of the free device memory with
# int-typed element counts (search_v2.cuh:799-805, 995-1001; size_a is an
# int, search_v2.cuh:29).  The harness parks memory so that the table holds
# 1.6e9 elements: 12 GiB of doubles for kNN, 6 GiB of ints for range -- a
# quarter below the int limit, so its kernels' int index arithmetic (thread
# ids over ql * n_l pairs) cannot wrap.
REF_BUDGET_GB = {"knn": 12.0, "range": 6.0}

WORKLOADS = {
    "cfg0": dict(kind="gmm", n=50_000, dim=300, comps=64, sigma=0.3, metric=2, max_h=5, queries=1000,
                 batches=[("knn", 8), ("range", ("quantile", 0.001, 1_000_000))], ref_queries=1000),
    "cfg1": dict(kind="words", n=1_000_000, dim=1, metric=6, max_h=6, queries=10_000,
                 batches=[("range", 1.0), ("range", 2.0), ("range", 3.0), ("knn", 16)], ref_queries=1000),
    "cfg2": dict(kind="gmm", n=1_000_000, dim=128, comps=256, sigma=0.2, metric=2, max_h=6, queries=10_000,
                 batches=[("knn", 8)], ref_queries=10_000),
    "cfg3": dict(kind="hot", n=10_000_000, dim=2, metric=1, max_h=7, queries=100_000,
                 batches=[("range", ("quantile", 0.0001, 2_000_000))], ref_queries=10_000),
    "cfg4": dict(kind="gmm", n=1_000_000, dim=300, comps=64, sigma=0.3, metric=2, max_h=6, queries=0,
                 batches=[("update", ("quantile", 0.001, 1_000_000))], ref_queries=0),
}
METRIC_NAME = {0: "Linf", 1: "L1", 2: "L2", 5: "angle", 6: "edit"}


def measured_peaks_all():
    """Roofline denominators: the driver-measured copy bandwidth and burst bf16
    GEMM throughput of this pool's B200s, else the pool's earlier figures."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "kind": "measured"}
    return {"hbm_gbs": HBM_FALLBACK_GBS, "bf16_tflops": BF16_FALLBACK_TFLOPS, "kind": "fallback"}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0=None, t1=None):
        """Median SM clock and the throttle reasons seen in [t0, t1] (host
        wall-clock seconds; the whole sampling when None)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if (t0 is not None and ts < t0) or (t1 is not None and ts > t1):
                continue
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ workloads

def spec(args) -> dict:
    """The workload's definition with the command-line overrides applied."""
    w = dict(WORKLOADS[args.workload])
    for key in ("n", "dim", "queries", "max_h"):
        v = getattr(args, key, None)
        if v is not None:
            w[key] = v
    if args.workload == "cfg2":
        if args.op == "range":
            w["batches"] = [("range", ("quantile", args.range_quantile, 20_000))]
        elif args.k_mix:
            w["batches"] = [("knn", k) for k in K_MIX]
        else:
            w["batches"] = [("knn", args.k)]
    if args.ref_queries is not None:
        w["ref_queries"] = args.ref_queries
    return w


def workload_name(args, w=None) -> str:
    w = w or spec(args)
    if w["kind"] == "words":
        base = f"words{w['n'] // 1000}k_edit"
    elif w["kind"] == "hot":
        base = f"hotspots{w['n'] // 1000}k_d{w['dim']}_{METRIC_NAME[w['metric']].lower()}"
    else:
        base = f"gmm{w['n'] // 1000}k_d{w['dim']}_{METRIC_NAME[w['metric']].lower()}"
    ops = sorted({op for op, _ in w["batches"]})
    tail = "_".join(ops)
    if args.workload == "cfg2" and args.k_mix and args.op == "knn":
        tail += "_kmix"
    return f"{base}_{tail}"


def make_data(w, seed):
    """-> (rows | None, (strs, lens) | None)."""
    from gts_b200 import datagen as G
    if w["kind"] == "gmm":
        return G.gmm_rows(w["n"], w["dim"], w["comps"], w["sigma"], seed=seed), None
    if w["kind"] == "hot":
        return G.hotspot_points(w["n"], seed), None
    return None, G.word_strings(w["n"], seed)


def resolve_param(op, param, w, rows, seed):
    """A batch parameter: k, a radius, or ("quantile", q, pairs) -> the radius
    at the q-quantile of that many seeded random pair distances."""
    from gts_b200 import datagen as G
    if isinstance(param, tuple) and param[0] == "quantile":
        return float(np.float32(G.quantile_radius(w["metric"], param[1], param[2], seed + 5, rows=rows)))
    return param


def make_batches(args, w, rows, n_queries):
    """[(op, k or r, query positions)] of one step.  A batch is one call of
    the search (the reference takes one k or r per run).  cfg2 --k-mix draws
    each query's k uniformly from {1, 8, 32, 64} (seeded)."""
    out = []
    if args.workload == "cfg2" and args.k_mix and args.op == "knn":
        ks = np.random.default_rng(args.seed + 99).choice(np.array(K_MIX), size=n_queries)
        return [("knn", k, np.nonzero(ks == k)[0]) for k in K_MIX if (ks == k).any()]
    for op, p in w["batches"]:
        out.append((op, resolve_param(op, p, w, rows, args.seed), np.arange(n_queries)))
    return out


def k_groups(args, n_queries):
    """(k, query positions) batches of a kNN step of the headline workload."""
    if not args.k_mix:
        return [(args.k, np.arange(n_queries))]
    ks = np.random.default_rng(args.seed + 99).choice(np.array(K_MIX), size=n_queries)
    return [(k, np.nonzero(ks == k)[0]) for k in K_MIX if (ks == k).any()]


def config_dict(args, world, w=None, batches=None):
    w = w or spec(args)
    c = {"workload": workload_name(args, w), "n": w["n"], "dim": w["dim"],
         "metric": METRIC_NAME[w["metric"]], "queries_per_gpu": w["queries"],
         "tree_order": 10, "max_size": 20, "max_h": w["max_h"], "form": args.form,
         "parallelism": f"query-sharded replicas x{world}",
         "l2_flush": ("yes: 256 MB buffer written before every step" if needs_flush(w)
                      else "no (data set larger than the 126 MB L2)")}
    if batches is not None:
        c["batches"] = [{"op": op, ("k" if op == "knn" else "radius"): p, "queries": len(sel)}
                        for op, p, sel in batches]
    if args.workload == "cfg2" and args.op == "range":
        c["range_quantile"] = args.range_quantile
        c["radius"] = getattr(args, "radius", None)
    if args.workload == "cfg2" and args.op == "knn":
        c["k"] = "uniform over {1, 8, 32, 64}, one batch per k" if args.k_mix else args.k
    return c


def needs_flush(w) -> bool:
    row = 109 + 4 if w["metric"] == 6 else 4 * w["dim"]
    return 2 * w["n"] * row < 126e6


def ref_result_path(args, w) -> str:
    key = f"{workload_name(args, w)}_n{w['n']}_d{w['dim']}_q{w['queries']}_s{args.seed}"
    return os.path.join(tempfile.gettempdir(), f"gts_ref_{key}.npz")


def kth_quantum(qnum: int) -> float:
    """Largest distance error of the reference's kNN sort code
    dist / INFI_DIS + qid * DIS_CODE (search_v2.cuh:541-542): one double ulp
    at the largest code of the batch, times INFI_DIS, with a factor 2."""
    code = max(1, qnum) * 100.0 + 1.0
    return float(np.spacing(np.float64(code)) * 10000.0 * 2.0)


# ------------------------------------------------------------------ reference arm

def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    drv = os.path.join(ROOT, "oracle", "_ref", "gts_ref_driver")
    from gts_b200 import datagen as G
    from gts_b200 import replicas as R
    w = spec(args)
    base = {"impl": "reference", "metric": metric_name(w), "unit": unit_name(w), "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True}
    if w["batches"][0][0] == "update":
        return run_reference_update(args, w, base, drv)
    rows, words = make_data(w, args.seed)
    qids = G.query_ids(w["n"], w["queries"], seed=R.rank_query_seed(args.seed, 0))
    batches = make_batches(args, w, rows, len(qids))
    base["config"] = config_dict(args, 1, w, batches)
    if not os.path.exists(drv):
        print(json.dumps({**base, "unavailable": "reference CUDA build oracle/_ref/gts_ref_driver is not built"}))
        return 0
    nref = min(w["ref_queries"], len(qids))
    t_total, wall, build_s, nq_total = 0.0, 0.0, 0.0, 0
    saved = {}
    per_batch = []
    repeat = args.warmup + args.steps
    with tempfile.TemporaryDirectory() as tmp:
        if w["metric"] == 6:
            dpath = os.path.join(tmp, "data.txt")
            G.write_data_text(dpath, 6, strs=words[0], lens=words[1])
        else:
            dpath = os.path.join(tmp, "data.bin")
            G.write_data_bin(dpath, w["metric"], rows)
        for bi, (op, p, sel) in enumerate(batches):
            # cfg2 --k-mix: one reference run per k over all of that k's queries
            sub = sel if (args.workload == "cfg2" and args.k_mix) else sel[:nref]
            qpath = os.path.join(tmp, f"q{bi}.txt")
            G.write_queries(qpath, qids[sub])
            out = os.path.join(tmp, f"res{bi}.txt")
            code, param = ("0", str(int(p))) if op == "knn" else ("1", repr(float(p)))
            dump = os.path.join(tmp, f"res{bi}.bin")
            cmd = [drv, dpath, qpath, code, param, out, "--order", "10", "--max-size", "20",
                   "--max-h", str(w["max_h"]), "--budget-gb", str(REF_BUDGET_GB[op]),
                   "--repeat", str(repeat), "--dump-res", dump]
            t0 = time.time()
            pr = subprocess.run(cmd, capture_output=True, text=True, timeout=args.ref_timeout)
            wall += time.time() - t0
            lines = [ln for ln in pr.stdout.splitlines() if ln.startswith("{")]
            if pr.returncode != 0 or not lines:
                print(json.dumps({**base, "unavailable": f"reference run failed rc={pr.returncode}: "
                                  f"{(pr.stderr or pr.stdout)[-300:]!r}"}))
                return 0
            info = json.loads(lines[-1])
            runs = info["search_runs"]
            t = statistics.mean(runs[min(args.warmup, len(runs) - 1):])
            t_total += t
            nq_total += len(sub)
            build_s = info["build_s"]
            # the reference's res / res_dis arrays as they are in memory (the
            # result file prints them with %f, 6 decimals)
            saved[f"pos{bi}"] = sub
            saved[f"val{bi}"] = np.fromfile(dump, dtype=np.int32 if op == "range" else np.float32)
            if len(saved[f"val{bi}"]) != len(sub):
                print(json.dumps({**base, "unavailable": f"reference result dump holds {len(saved[f'val{bi}'])} "
                                                         f"values for {len(sub)} queries"}))
                return 0
            per_batch.append({"op": op, ("k" if op == "knn" else "radius"): p, "queries": len(sub),
                              "queries_per_s": len(sub) / t, "search_s": t})
    value = nq_total / t_total
    sample = (f"reference CUDA build ({', '.join(sorted({'searchIndexKnnV2' if op == 'knn' else 'searchIndexRnnV2' for op, _, _ in batches}))}) "
              f"on the B200, {nq_total} of the step's {sum(len(s) for _, _, s in batches)} queries "
              f"({nref} per batch), list-table budget {REF_BUDGET_GB} GB; one host thread drives it")
    line = {**base, "value": value, "ms_per_step": t_total * 1e3, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64" if w["metric"] != 6 else "int",
            "data": data_desc(w), "build_s": build_s, "wall_s": wall, "batches": per_batch,
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": 1, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    np.savez(ref_result_path(args, w), **saved)
    print(json.dumps(line))
    return 0


def run_reference_update(args, w, base, drv):
    """The reference's updateIndexRnn (update.cuh:449-638) on a prefix of the
    stream (it rebuilds the whole index every MAX_IN_SIZE inserts)."""
    from gts_b200 import datagen as G
    rows, _ = make_data(w, args.seed)
    r = resolve_param("update", w["batches"][0][1], w, rows, args.seed)
    nops = min(args.ops, args.ref_ops)
    flags, ids = G.update_stream(w["n"], args.ops, args.seed + 3000, 10)
    flags, ids = flags[:nops], ids[:nops]
    base["config"] = update_config(args, w, r, nops)
    if not os.path.exists(drv):
        print(json.dumps({**base, "unavailable": "reference CUDA build oracle/_ref/gts_ref_driver is not built"}))
        return 0
    with tempfile.TemporaryDirectory() as tmp:
        dpath = os.path.join(tmp, "data.bin")
        G.write_data_bin(dpath, 2, rows)
        upath = os.path.join(tmp, "u.txt")
        G.write_updates(upath, flags, ids)
        out = os.path.join(tmp, "res.txt")
        cmd = [drv, dpath, upath, "2", repr(float(r)), out, "--order", "10", "--max-size", "20",
               "--max-h", str(w["max_h"]), "--max-in-size", "10", "--budget-gb", "0"]
        t0 = time.time()
        pr = subprocess.run(cmd, capture_output=True, text=True, timeout=args.ref_timeout)
        wall = time.time() - t0
        lines = [ln for ln in pr.stdout.splitlines() if ln.startswith("{")]
        if pr.returncode != 0 or not lines:
            print(json.dumps({**base, "unavailable": f"reference run failed rc={pr.returncode}: "
                              f"{(pr.stderr or pr.stdout)[-300:]!r}"}))
            return 0
        info = json.loads(lines[-1])
        vals = np.array([int(v) for v in open(out).read().split("\n")[2].split()], np.int32)
    t = info["search_s"]   # the whole updateIndexRnn call (its ops, rebuilds and queries)
    value = nops / t
    np.savez(ref_result_path(args, w), pos0=np.arange(len(vals)), val0=vals, nops=np.array([nops]))
    print(json.dumps({**base, "value": value, "ms_per_step": t * 1e3, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": data_desc(w),
                      "build_s": info["build_s"], "wall_s": wall,
                      "cpu_baseline": {"value": value, "unit": "ops/s", "cores": 1, "kind": "reference",
                                       "sample": f"reference CUDA build (updateIndexRnn) on the B200, the "
                                                 f"first {nops} of the {args.ops} operations; one host thread"},
                      "e2e": {"value": value, "unit": "ops/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))
    return 0


def metric_name(w) -> str:
    ops = {op for op, _ in w["batches"]}
    if ops == {"update"}:
        return "stream-update operations/s"
    if ops == {"knn"}:
        return "exact kNN queries/s"
    if ops == {"range"}:
        return "exact range queries/s"
    return "exact kNN + range queries/s"


def unit_name(w) -> str:
    return "ops/s" if w["batches"][0][0] == "update" else "queries/s"


def data_desc(w) -> str:
    what = {"gmm": "Gaussian mixture", "words": "Zipf-letter words", "hot": "2-D hotspots"}[w["kind"]]
    return f"synthetic (seeded {what}; the paper's data sets are absent)"


def update_config(args, w, r, nops):
    return {"workload": f"gmm{w['n'] // 1000}k_d{w['dim']}_l2_update", "n": w["n"], "dim": w["dim"],
            "metric": "L2", "ops": nops, "mix": "45% insert / 45% delete / 10% range query",
            "radius": r, "max_in_size": 10, "tree_order": 10, "max_size": 20, "max_h": w["max_h"],
            "parallelism": "one GPU", "l2_flush": "no (1.2 GB data set larger than the 126 MB L2)"}


# ------------------------------------------------------------------ our arm

def cpu_baseline(w, rows, words, qids, batches, sample, got):
    """Exact multi-threaded brute force (reference leaf arithmetic) on the
    host, on the leading queries of each batch (sample split evenly)."""
    from oracle import oracle as O
    ds = O.Dataset(w["metric"], rows) if words is None else O.Dataset(6, strs=words[0], lens=words[1])
    cores = os.cpu_count() or 1
    per = max(1, sample // len(batches))
    n, agree, dt = 0, 0, 0.0
    for bi, (op, p, sel) in enumerate(batches):
        sub = sel[:per]
        t0 = time.perf_counter()
        if op == "range":
            ans = O.range_brute(ds, qids[sub], p, nthreads=cores)
        else:
            ans, _, _ = O.knn_brute(ds, qids[sub], int(p), nthreads=cores)
        dt += time.perf_counter() - t0
        agree += int((ans == got[bi][:len(sub)]).sum())
        n += len(sub)
    return {"value": n / dt, "unit": "queries/s", "cores": cores, "kind": "port",
            "sample": f"{n} of the {sum(len(s) for _, _, s in batches)} queries ({per} per batch), exact "
                      f"brute force over all {w['n']} objects in the reference's leaf arithmetic, {cores} threads",
            "agrees_with_gpu": f"{agree}/{n}"}


def compare_with_reference(args, w, batches, got, rows=None, words=None, qids=None):
    """Every answer the reference arm saved for this workload against ours:
    counts exactly, k-th distances exactly or within the reference's sort-code
    quantum (a near-tie its quantised code swapped).  Where they differ, the
    oracle's exact brute force (given the data) says which side is right, on
    up to 64 of those queries."""
    path = ref_result_path(args, w)
    if not os.path.exists(path):
        return {"checked": 0, "note": "no reference answers saved on this machine for this workload "
                                      "(run bench.py --impl reference first)"}
    ref = np.load(path)
    checked, exact, within, worst = 0, 0, 0, 0.0
    differ = []   # (batch, op, param, query position, ours, reference's)
    for bi, (op, p, sel) in enumerate(batches):
        if f"pos{bi}" not in ref:
            continue
        pos, val = ref[f"pos{bi}"], ref[f"val{bi}"]
        lookup = {int(s): j for j, s in enumerate(sel)}
        mine = np.array([got[bi][lookup[int(x)]] for x in pos])
        checked += len(pos)
        if op == "range":
            ok = mine == val
            exact += int(ok.sum())
            within += int(ok.sum())
        else:
            q = kth_quantum(len(pos))
            diff = np.abs(mine.astype(np.float64) - val.astype(np.float64))
            ok = diff <= q
            exact += int((diff == 0).sum())
            within += int(ok.sum())
            worst = max(worst, float(diff.max()) if len(diff) else 0.0)
        for j in np.nonzero(~ok)[0]:
            differ.append((bi, op, p, int(pos[j]), mine[j], val[j]))
    out = {"checked": checked, "identical": exact, "within_sort_code_quantum": within,
           "max_abs_kth_diff": worst, "agrees": within == checked}
    if differ and qids is not None and (rows is not None or words is not None):
        out["differences_by_oracle"] = adjudicate(w, rows, words, qids, differ[:64])
    return out


def adjudicate(w, rows, words, qids, differ):
    """The oracle's exact brute force on the queries where this build and the
    reference disagree: how many of them each side answers exactly."""
    from oracle import oracle as O
    ds = O.Dataset(w["metric"], rows) if words is None else O.Dataset(6, strs=words[0], lens=words[1])
    ours = theirs = 0
    examples = []
    for bi, op, p, qpos, mine, val in differ:
        q = np.array([qids[qpos]], np.int32)
        truth = (O.range_brute(ds, q, p)[0] if op == "range" else O.knn_brute(ds, q, int(p))[0][0])
        ours += int(mine == truth)
        theirs += int(val == truth)
        if len(examples) < 5:
            examples.append({"query": int(q[0]), "op": op, "param": p, "ours": mine.item(), "reference": val.item(),
                             "exact": truth.item()})
    return {"examined": len(differ), "ours_exact": ours, "reference_exact": theirs, "examples": examples}


def flush_l2(torch, dev, buf):
    if buf is not None:
        buf.zero_()


def run_gts(args):
    import torch
    import torch.distributed as dist

    import gts_b200 as gts
    from gts_b200 import datagen as G
    from gts_b200 import replicas as R

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    w = spec(args)
    if w["batches"][0][0] == "update":
        return run_gts_update(args, w, world, rank, dev, stream)

    rows, words = make_data(w, args.seed)
    qids = G.query_ids(w["n"], w["queries"], seed=R.rank_query_seed(args.seed, rank))
    batches = make_batches(args, w, rows, len(qids))
    if args.workload == "cfg2" and args.op == "range":
        args.radius = batches[0][1]
    form_name = args.form
    form = {"fast": gts.FORM_FAST, "plain": gts.FORM_PLAIN, "plain-learned": gts.FORM_PLAIN_LEARNED}[form_name]
    params = gts.Params(max_h=w["max_h"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if words is not None:
        idx = gts.Index(None, 6, strs=words[0], lens=words[1], params=params)
        idx.set_stream(stream.cuda_stream)
    else:
        d_rows = torch.from_numpy(rows).to(dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        idx = gts.Index.from_device(d_rows.data_ptr(), w["n"], w["dim"], w["metric"], params=params,
                                    stream=stream.cuda_stream)
        torch.cuda.synchronize()
        del d_rows
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    # the tensor-core form's block order and filter records (built once per
    # index; without this call the first fast query builds them)
    t0 = time.perf_counter()
    prepared = idx.prepare(form, stream.cuda_stream)
    torch.cuda.synchronize()
    prepare_s = time.perf_counter() - t0
    index_bytes = idx.info["device_bytes"]
    has_knn = any(op == "knn" for op, _, _ in batches)
    fast_ok = w["metric"] == 2 and w["dim"] <= 320
    learn = None
    if form_name in ("fast", "plain-learned") and not args.no_learn and has_knn and fast_ok:
        # learned radius: exact radii of 200,000 objects from the index
        # itself, trained on the device before the timed region
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        learn = idx.learn_radius(n_train=args.train, k_max=64, epochs=12, seed=args.seed)
        torch.cuda.synchronize()
        learn["train_s"] = time.perf_counter() - t0
        learn["n_train"] = args.train
    if form_name == "plain-learned" and any(op == "range" for op, _, _ in batches):
        raise SystemExit("--form plain-learned takes kNN workloads")
    groups = []
    for op, p, sel in batches:
        groups.append({"op": op, "p": p, "sel": sel,
                       "q": torch.from_numpy(np.ascontiguousarray(qids[sel])).to(dev),
                       "out": torch.empty(len(sel), dtype=torch.int32 if op == "range" else torch.float32,
                                          device=dev)})
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev) if needs_flush(w) else None

    def run_group(g):
        if g["op"] == "range":
            idx.range_device(g["q"].data_ptr(), len(g["sel"]), g["p"], g["out"].data_ptr(),
                             stream=stream.cuda_stream, form=form if form != gts.FORM_PLAIN_LEARNED else gts.FORM_PLAIN)
        else:
            idx.knn_device(g["q"].data_ptr(), len(g["sel"]), int(g["p"]), g["out"].data_ptr(), form=form,
                           stream=stream.cuda_stream)

    def step():
        for g in groups:
            run_group(g)

    if form_name == "fast" and args.fast_filter != "auto":
        idx.fast_range_variant(0 if args.fast_filter == "block" else 1)
    pin_seed = learn is not None and form_name == "fast" and args.learned_seed != "auto"
    if pin_seed or (form_name == "fast" and args.fast_filter != "auto"):
        step()   # tunes the configuration for each k, then the seed choice or the filter is pinned
        torch.cuda.synchronize()
        for g in groups:
            if g["op"] == "knn":
                c = idx.fast_config(int(g["p"]))
                learned = c["learned_seed"] if not pin_seed else args.learned_seed == "on"
                blk = c["by_block"] if args.fast_filter == "auto" else args.fast_filter == "block"
                streamed = c["streamed"] and not blk
                idx.set_fast_config(int(g["p"]), learned, c["col_groups"], c["item_blocks"], streamed, blk)
    clocks = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        flush_l2(torch, dev, flush)
        step()
    torch.cuda.synchronize()
    # work counters of one step (the library keeps those of its last call)
    stats = {}
    for g in groups:
        run_group(g)
        torch.cuda.synchronize()
        for key, v in idx.search_stats().items():
            stats[key] = stats.get(key, 0) + v
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    use_fast_timer = form_name == "fast" and fast_ok
    if use_fast_timer:
        idx.filter_timing(reset=True)
    if args.profile:
        torch.cuda.profiler.start()
    launches0 = idx.kernel_launches()
    wall0 = time.time()
    for i in range(args.steps):
        flush_l2(torch, dev, flush)
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    wall1 = time.time()
    launches = idx.kernel_launches() - launches0
    filter_ms, filter_launches = idx.filter_timing() if use_fast_timer else (0.0, 0)
    if args.profile:
        torch.cuda.profiler.stop()
    # nvidia-smi samples every 100 ms: when the timed steps are shorter than
    # that, the same step keeps running (untimed) until 0.3 s have passed so
    # the clock record covers this load
    while time.time() - wall0 < 0.3:
        step()
        torch.cuda.synchronize()
    wall2 = time.time()
    time.sleep(0.15)   # let the last sample land
    clocks.__exit__(None, None, None)
    clock_summary = clocks.summary(wall0, wall2)
    clock_summary["window_s"] = round(wall2 - wall0, 3)
    clock_summary["timed_s"] = round(wall1 - wall0, 3)
    per_step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(per_step_ms)
    if world > 1:
        total_ms = R.max_over_ranks(total_ms, dist, dev)
        dist.barrier()
    ms_per_step = total_ms / args.steps
    Q = sum(len(g["sel"]) for g in groups)
    value = world * Q * args.steps / (total_ms / 1e3)
    got = [g["out"].cpu().numpy() for g in groups]

    # end to end through the host-buffer API: H2D of the query ids from pinned
    # memory and D2H of the answers inside every timed call
    def host_call(g):
        if g["op"] == "range":
            return idx.range(g["h_q"], g["p"], form=form if form != gts.FORM_PLAIN_LEARNED else gts.FORM_PLAIN)
        return idx.knn(g["h_q"], int(g["p"]), form=form)

    for g in groups:
        g["h_q"] = torch.from_numpy(np.ascontiguousarray(qids[g["sel"]])).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        for g in groups:
            host_call(g)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_s = 0.0
    for _ in range(args.steps):
        flush_l2(torch, dev, flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs = [host_call(g) for g in groups]
        e2e_s += time.perf_counter() - t0
    if world > 1:
        e2e_s = R.max_over_ranks(e2e_s, dist, dev)
    e2e = {"value": world * Q * args.steps / e2e_s, "unit": "queries/s",
           "h2d_bytes_per_step": int(sum(g["h_q"].nbytes for g in groups)),
           "d2h_bytes_per_step": int(sum(x.nbytes for x in outs))}
    for g, x, y in zip(groups, outs, got):
        assert np.array_equal(x, y), "host-buffer and device-buffer paths disagree"

    peaks = measured_peaks_all()
    # the filter the step ran: block-stationary (per k, as tuned; range counts
    # at widths up to 128) or the tile filter
    by_block = use_fast_timer and all(
        idx.fast_config(int(g["p"]))["by_block"] if g["op"] == "knn"
        else (idx.fast_range_variant() == 0 and w["dim"] <= 128) for g in groups)
    roofline = make_roofline(args, w, groups, stats, per_step_ms, total_ms, filter_ms, filter_launches,
                             use_fast_timer, peaks, by_block)
    line = {"metric": metric_name(w), "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("bf16/f32/f64" if use_fast_timer else "f32/f64") if w["metric"] != 6 else "int",
            "data": data_desc(w),
            "config": config_dict(args, world, w, batches),
            "build_s": build_s, "prepare_s": prepare_s if prepared else 0.0,
            "index_device_bytes": index_bytes, "learned_radius": learn,
            "autotune": autotune_record(idx, groups, use_fast_timer),
            "roofline": roofline,
            "e2e": e2e, "gpu_launches": launches, "clocks": clock_summary}
    if len(groups) > 1:
        # per-batch rates from one more step, each batch bracketed by events
        per = []
        for g in groups:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush_l2(torch, dev, flush)
            a.record(stream)
            run_group(g)
            b.record(stream)
            torch.cuda.synchronize()
            per.append({"op": g["op"], ("k" if g["op"] == "knn" else "radius"): g["p"],
                        "queries": len(g["sel"]), "queries_per_s": len(g["sel"]) / (a.elapsed_time(b) / 1e3)})
        line["batches"] = per
    if rank == 0:
        line["agrees_with_reference"] = compare_with_reference(args, w, batches, got, rows, words, qids)
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        line["cpu_baseline"] = cpu_baseline(w, rows, words, qids, batches, args.cpu_sample, got)
    if rank == 0:
        print(json.dumps(line))
    idx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def autotune_record(idx, groups, fast):
    if fast:
        ks = sorted({int(g["p"]) for g in groups if g["op"] == "knn"})
        rec = {str(k): idx.fast_config(k) for k in ks}
        if len(ks) == 1:
            rec = rec[str(ks[0])]
        return rec
    return {"threads_per_query_cta": {m: idx.plain_threads(i) for i, m in enumerate(("knn", "range"))}}


def make_roofline(args, w, groups, stats, per_step_ms, total_ms, filter_ms, filter_launches, fast, peaks,
                  by_block=False):
    # DRAM traffic of the dominant kernel per launch: the ncu capture's bytes
    # per unit (operand block for the filter, leaf object for the traversal)
    # times the units this run processed per launch
    per_unit = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            per_unit = json.load(f)
    d = w["dim"]
    step_ms = statistics.mean(per_step_ms)
    if not fast:
        # every leaf row and pivot row a query reads, plus its own row and
        # result; a string row is its 109 bytes plus its 4-byte length
        row = 4 * d if w["metric"] != 6 else 113
        alg_bytes = row * (stats["objects"] + stats["pivots"]) + sum(
            len(g["sel"]) * (row + (4 if g["op"] == "range" else 8 * int(g["p"]))) for g in groups)
        achieved = alg_bytes / (step_ms / 1e3) / 1e9
        traffic = None
        if "k_search" in per_unit and w["metric"] == 2:
            traffic = per_unit["k_search"]["dram_bytes_per_object"] * stats["objects"] * d / 128
        Q = sum(len(g["sel"]) for g in groups)
        return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peaks["kind"],
                "kernel": "k_search (the plain traversal; the step's launches of it, one per batch)",
                "alg_bytes_per_step": alg_bytes,
                "per_query": {"leaf_objects": stats["objects"] / Q, "pivots": stats["pivots"] / Q,
                              "exact_rechecks": stats["exact"] / Q}}
    Q = sum(len(g["sel"]) for g in groups)
    kp = (d + 63) // 64 * 64
    per_step = max(1, filter_launches // max(1, args.steps))
    kernel_ms = filter_ms / max(1, filter_launches)
    per_query = {"blocks": stats["blocks"] / Q, "appended": stats["appended"] / Q,
                 "exact_rechecks": stats["exact"] / Q,
                 "fallback_queries": stats["fallback"], "passes": stats["passes"]}
    if by_block:
        # HBM: every item streams its block's record (BF16 operand rows of the
        # 128 objects, the centre rows, w and |d|) once; a block needed by
        # more than 32 queries is one item per 32 of them
        items = stats["blocks"] / per_step
        alg = stats["bytes"] / per_step
        achieved = alg / (kernel_ms / 1e3) / 1e9
        traffic = None
        if "k_fast_blk" in per_unit:
            traffic = per_unit["k_fast_blk"]["dram_bytes_per_item"] * items
        return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peaks["kind"],
                "kernel": "k_fast_blk", "kernel_ms_per_launch": kernel_ms, "launches_per_step": per_step,
                "kernel_share_of_step": filter_ms / total_ms,
                "items_per_launch": items, "record_bytes_per_launch": alg,
                "pairs_per_query": stats["queries"] / Q,
                "record_bytes_per_item": (stats["bytes"] / stats["blocks"]) if stats["blocks"] else None,
                "per_query": per_query,
                "block_pairs_kept": (stats["blocks"] / stats["tested"]) if stats["tested"] else None}
    # tensor pipe: every streamed block is one 128 x 144 x Kp MMA chain for
    # the BF16 high part and one for the low part of the queries, timed on
    # the device around every filter launch (CUDA events on the launching
    # stream); one step runs the filter once per batch, plus once per
    # re-answer stage when queries fail
    flops = stats["blocks"] * 2 * 128 * 144 * kp * 2 / per_step
    achieved = flops / (kernel_ms / 1e3) / 1e12
    traffic = None
    if "k_fast_tile" in per_unit:
        traffic = per_unit["k_fast_tile"]["dram_bytes_per_block"] * stats["blocks"] / per_step
    streamed = stats["bytes"] / per_step
    return {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"],
            "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"], "traffic": traffic,
            "peak_kind": peaks["kind"], "kernel": "k_fast_tile",
            "kernel_ms_per_launch": kernel_ms, "launches_per_step": per_step,
            "kernel_share_of_step": filter_ms / total_ms,
            "mma_flops_per_launch": flops,
            "streamed_bytes_per_launch": streamed,
            "streamed_gbs": streamed / (kernel_ms / 1e3) / 1e9,
            "streamed_hbm_frac": streamed / (kernel_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
            "per_query": per_query,
            "block_pairs_kept": (stats["blocks"] / stats["tested"]) if stats["tested"] else None}


def run_gts_update(args, w, world, rank, dev, stream):
    """The stream-update workload: the whole op stream through
    gts_update_run (host buffers in, counts out; the call is the timed unit),
    on a fresh index per step (the call rewrites the index)."""
    import torch

    import gts_b200 as gts
    from gts_b200 import datagen as G
    if args.new_rows:
        # inserts bring new samples of the same mixture: the data rows are the
        # first n of one mixture draw, the inserted rows the rest
        flags, ids = G.update_stream_new_rows(w["n"], args.ops, args.seed + 3000, 10)
        n_new = int((flags == 0).sum())
        both = G.gmm_rows(w["n"] + n_new, w["dim"], w["comps"], w["sigma"], seed=args.seed)
        rows, new_rows = both[:w["n"]], both[w["n"]:]
    else:
        rows, _ = make_data(w, args.seed)
        flags, ids = G.update_stream(w["n"], args.ops, args.seed + 3000, 10)
        new_rows = None
    r = resolve_param("update", w["batches"][0][1], w, rows, args.seed)
    params = gts.Params(max_h=w["max_h"], max_in_size=10)
    d_rows = torch.from_numpy(rows).to(dev)
    torch.cuda.synchronize()
    times, search_s, update_s, builds = [], [], [], []
    counts = None
    launches = 0
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))).__enter__()
    wall0 = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        idx = gts.Index.from_device(d_rows.data_ptr(), w["n"], w["dim"], 2, params=params,
                                    stream=stream.cuda_stream)
        torch.cuda.synchronize()
        builds.append(time.perf_counter() - t0)
        l0 = idx.kernel_launches()
        if i == args.warmup:
            wall0 = time.time()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        t0 = time.perf_counter()
        if new_rows is not None:
            c, ts, tu = idx.update_run_rows(flags, ids, new_rows, r)
        else:
            c, ts, tu = idx.update_run(flags, ids, r)
        b.record(stream)
        torch.cuda.synchronize()
        wall_call = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(a.elapsed_time(b) / 1e3)
            search_s.append(ts)
            update_s.append(tu)
            launches += idx.kernel_launches() - l0
        if counts is None:
            counts = c
        assert np.array_equal(c, counts), "update stream answers differ between steps"
        idx.close()
    wall1 = time.time()
    clocks.__exit__(None, None, None)
    clock_summary = clocks.summary(wall0, wall1)
    t = statistics.mean(times)
    value = args.ops / t
    line = {"metric": metric_name(w), "value": value, "unit": "ops/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": data_desc(w), "config": update_config(args, w, r, args.ops),
            "build_s": statistics.mean(builds), "query_ops": int((flags == 2).sum()),
            "search_s": statistics.mean(search_s), "update_s": statistics.mean(update_s),
            "e2e": {"value": value, "unit": "ops/s",
                    "h2d_bytes_per_step": int(flags.nbytes + ids.nbytes + (new_rows.nbytes if new_rows is not None else 0)),
                    "d2h_bytes_per_step": int(counts.nbytes),
                    "note": "gts_update_run takes host buffers: the timed call includes their copies"},
            "gpu_launches": launches // max(1, args.steps), "clocks": clock_summary}
    if new_rows is not None:
        # the reference cannot insert new rows: the oracle's exact
        # restatement checks a prefix of the stream
        from oracle import oracle as O
        pre = min(args.ops, args.oracle_ops)
        nq_pre = int((flags[:pre] == 2).sum())
        t0 = time.perf_counter()
        want = O.update_run_rows(O.Dataset(2, rows), 10, flags[:pre], ids[:pre], new_rows, r)
        line["agrees_with_oracle"] = {"ops": pre, "checked": nq_pre,
                                      "agrees": bool(np.array_equal(counts[:nq_pre], want)),
                                      "oracle_s": time.perf_counter() - t0}
        line["config"]["inserts"] = "new samples of the same mixture (gts_update_run_rows)"
        path = None
    else:
        path = ref_result_path(args, w)
    if path is None:
        pass
    elif os.path.exists(path):
        ref = np.load(path)
        vals = ref["val0"]
        line["agrees_with_reference"] = {"checked": len(vals), "identical": int((counts[:len(vals)] == vals).sum()),
                                         "agrees": bool(np.array_equal(counts[:len(vals)], vals)),
                                         "ops": int(ref["nops"][0])}
    else:
        line["agrees_with_reference"] = {"checked": 0, "note": "no reference answers saved on this machine"}
    if rank == 0:
        print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ launch

def relaunch_under_torchrun(args) -> int:
    """`--gpus N` (N > 1) without a torchrun environment: run this script
    again as N ranks on this node, one per GPU."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def run_dry(args):
    """--dry-run: the launch, rendezvous and max-over-ranks timing of the
    multi-rank path with no GPU work (gloo), for CPU tests."""
    import torch.distributed as dist

    from gts_b200 import replicas as R
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = R.max_over_ranks(1.0 + rank, dist if world > 1 else None)
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "max_over_ranks": t,
                          "workload": workload_name(args)}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cfg2")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gts", "reference"], default="gts")
    ap.add_argument("--form", choices=["fast", "plain", "plain-learned"], default="fast",
                    help="fast: tensor-core filter where the index allows it (L2, dim <= 128), else the "
                         "plain traversal; plain-learned: the plain traversal seeded by the trained radius")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--dim", type=int, default=None)
    ap.add_argument("--queries", type=int, default=None)
    ap.add_argument("--max-h", type=int, default=None)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--op", choices=["knn", "range"], default="knn",
                    help="cfg2 only -- range: range counts at the --range-quantile distance quantile")
    ap.add_argument("--range-quantile", type=float, default=0.001)
    ap.add_argument("--k-mix", action="store_true",
                    help="cfg2 only: k uniform over {1, 8, 32, 64} per query (one batch per k per step)")
    ap.add_argument("--ops", type=int, default=1_000_000, help="cfg4: operations in the stream")
    ap.add_argument("--ref-ops", type=int, default=2000, help="cfg4: operations the reference arm runs")
    ap.add_argument("--new-rows", action="store_true",
                    help="cfg4: inserts bring new mixture samples (the reference can only copy rows; "
                         "checked against the oracle on --oracle-ops operations)")
    ap.add_argument("--oracle-ops", type=int, default=400)
    ap.add_argument("--ref-queries", type=int, default=None,
                    help="queries per batch the reference arm runs (default: per workload)")
    ap.add_argument("--ref-timeout", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample", type=int, default=256)
    ap.add_argument("--no-learn", action="store_true",
                    help="fast form without the learned radius (own-block seeds only)")
    ap.add_argument("--train", type=int, default=200_000, help="learned-radius training samples")
    ap.add_argument("--learned-seed", choices=["auto", "on", "off"], default="auto",
                    help="fast form with a trained radius: let the autotuner choose the learned seed, "
                         "or force it on / off (the other tuned settings are kept)")
    ap.add_argument("--fast-filter", choices=["auto", "tile", "block"], default="auto",
                    help="fast form: the autotuner's filter per k, or pin the tile or the block-stationary filter "
                         "(range counts: the block filter where it fits unless tile)")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--dry-run", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args(argv)


def main():
    args = parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(args)
    if args.dry_run:
        return run_dry(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_gts(args)


if __name__ == "__main__":
    sys.exit(main())
