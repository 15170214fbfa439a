"""Benchmark: exact kNN queries/s on one B200 (GTS similarity-search path).

Workload (the headline configuration): 1,000,000 x 128 float32 vectors from a
256-component Gaussian mixture (sigma 0.2, seeded, synthetic: the paper's
data sets are not available), L2, 10,000 concurrent kNN queries with query
ids drawn from the data, k = 8; GTS tree with TREE_ORDER 10, MAX_SIZE 20,
MAX_H 6 (a perfect tree: 100,000 leaves of 10 objects).

One step = one batch of 10,000 queries through the search.  The data set
(512 MB) is larger than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gts|reference]
                    [--form fast|plain|plain-learned] [--k 8 | --k-mix]
                    [--queries 10000] [--n 1000000]

--k-mix runs the same data with each query's k drawn uniformly from
{1, 8, 32, 64}: one batch per k per step (the reference takes one k per run).
--op range times range counts instead, at the --range-quantile (0.001)
distance quantile of seeded random pairs.

--impl reference times the reference's own CUDA build (oracle/_ref, built
from the reference sources) through its entry points on the same workload
and prints the same JSON line with "impl": "reference".

Multi-GPU (torchrun, one rank per GPU): every rank holds a replica of the
index and answers its own 10,000 queries (weak scaling, no collective on the
data path); the time is the max over ranks.
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


def workload(args, rank=0):
    from gts_b200 import datagen as G
    rows = G.gmm_rows(args.n, args.dim, 256, 0.2, seed=args.seed)
    from gts_b200 import replicas as R
    qids = G.query_ids(args.n, args.queries, seed=R.rank_query_seed(args.seed, rank))
    if args.op == "range":
        # the radius at the given quantile of seeded random pair distances
        args.radius = float(np.float32(G.quantile_radius(2, args.range_quantile, 20000, args.seed + 5, rows=rows)))
    return rows, qids


K_MIX = (1, 8, 32, 64)


def k_groups(args, n_queries):
    """(k, query positions) batches of one step.  --k-mix draws each query's k
    uniformly from {1, 8, 32, 64} (seeded) and runs one batch per k, as the
    reference takes one k per run; otherwise one batch with --k."""
    if not args.k_mix:
        return [(args.k, np.arange(n_queries))]
    ks = np.random.default_rng(args.seed + 99).choice(np.array(K_MIX), size=n_queries)
    return [(k, np.nonzero(ks == k)[0]) for k in K_MIX if (ks == k).any()]


def config_dict(args, world):
    if args.op == "range":
        return {"workload": f"gmm{args.n // 1000}k_d{args.dim}_l2_range",
                "n": args.n, "dim": args.dim, "metric": "L2", "queries_per_gpu": args.queries,
                "range_quantile": args.range_quantile, "radius": getattr(args, "radius", None),
                "tree_order": 10, "max_size": 20, "max_h": args.max_h,
                "form": args.form + (" (bf16 filter, bound fixed at r^2)" if args.form == "fast" else ""),
                "parallelism": f"query-sharded replicas x{world}",
                "l2_flush": "no (512 MB data set > 126 MB L2)"}
    return {"workload": f"gmm{args.n // 1000}k_d{args.dim}_l2_knn" + ("_kmix" if args.k_mix else ""),
            "n": args.n, "dim": args.dim, "metric": "L2", "queries_per_gpu": args.queries,
            "k": ("uniform over {1, 8, 32, 64}, one batch per k" if args.k_mix else args.k),
            "tree_order": 10, "max_size": 20, "max_h": args.max_h,
            "form": args.form + ("" if args.form != "fast" else
                                 (" (block-pruned bf16 filter)" if args.no_learn else
                                  " (learned radius trained + block-pruned bf16 filter; " +
                                  {"auto": "the autotuner decides per k whether the learned seed is used)",
                                   "on": "learned seed forced on)",
                                   "off": "learned seed forced off)"}[args.learned_seed])),
            "parallelism": f"query-sharded replicas x{world}",
            "l2_flush": "no (512 MB data set > 126 MB L2)"}


# ------------------------------------------------------------------ reference arm

def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    drv = os.path.join(ROOT, "oracle", "_ref", "gts_ref_driver")
    from gts_b200 import datagen as G
    rows, qids = workload(args)
    rng = args.op == "range"
    base = {"impl": "reference", "metric": "exact range queries/s" if rng else "exact kNN queries/s",
            "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "config": config_dict(args, 1)}
    if not os.path.exists(drv):
        print(json.dumps({**base, "unavailable": "reference CUDA build oracle/_ref/gts_ref_driver is not built"}))
        return 0
    ref_kth = np.zeros(len(qids), np.int32 if rng else np.float32)
    t, wall, build_s = 0.0, 0.0, 0.0
    with tempfile.TemporaryDirectory() as tmp:
        dpath = os.path.join(tmp, "data.bin")
        G.write_data_bin(dpath, 2, rows)
        # one reference run per k (it takes one k per run); a step is all of them
        groups = [(0, np.arange(len(qids)))] if rng else k_groups(args, len(qids))
        for k, sel in groups:
            qpath = os.path.join(tmp, f"q{k}.txt")
            G.write_queries(qpath, qids[sel])
            out = os.path.join(tmp, f"res{k}.txt")
            op, param = ("1", repr(args.radius)) if rng else ("0", str(k))
            cmd = [drv, dpath, qpath, op, param, out, "--order", "10", "--max-size", "20",
                   "--max-h", str(args.max_h), "--budget-gb", "6",
                   "--repeat", str(args.warmup + args.steps)]
            t0 = time.time()
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=3000)
            wall += time.time() - t0
            lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
            if p.returncode != 0 or not lines:
                print(json.dumps({**base, "unavailable": f"reference run failed rc={p.returncode}: "
                                  f"{(p.stderr or p.stdout)[-300:]!r}"}))
                return 0
            info = json.loads(lines[-1])
            t += statistics.mean(info["search_runs"][args.warmup:])
            build_s += info["build_s"]
            vals = open(out).read().split("\n")[2].split()
            ref_kth[sel] = (np.array([int(v) for v in vals], np.int32) if rng
                            else np.array([float(v) for v in vals], np.float32))
        value = args.queries / t
    line = {**base, "value": value, "ms_per_step": t * 1e3, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian mixture)",
            "build_s": build_s, "wall_s": wall,
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": 1, "kind": "reference",
                             "sample": f"reference CUDA build ({'searchIndexRnnV2' if rng else 'searchIndexKnnV2'}) on the B200, "
                                       f"{args.queries} queries per step, 6 GB list-table budget; "
                                       f"one host thread drives it"},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    np.save(os.path.join(tempfile.gettempdir(), "gts_ref_kth.npy"), ref_kth)
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm

def cpu_baseline(rows, qids, groups, sample, kth_gpu, radius=None):
    """Exact multi-threaded brute force (reference leaf arithmetic) on the host,
    on the leading queries of each k batch (sample split evenly)."""
    from oracle import oracle as O
    ds = O.Dataset(2, rows)
    cores = os.cpu_count() or 1
    per = max(1, sample // len(groups))
    n, agree, dt = 0, 0, 0.0
    for g in groups:
        sel = g["sel"][:per]
        t0 = time.perf_counter()
        if radius is not None:
            kth = O.range_brute(ds, qids[sel], radius, nthreads=cores)
        else:
            kth, _, _ = O.knn_brute(ds, qids[sel], g["k"], nthreads=cores)
        dt += time.perf_counter() - t0
        agree += int((kth == kth_gpu[sel]).sum())
        n += len(sel)
    return {"value": n / dt, "unit": "queries/s", "cores": cores, "kind": "port",
            "sample": f"{n} of the {len(qids)} queries, exact brute force over all "
                      f"{len(rows)} rows in the reference's {'F32 range' if radius is not None else 'F64 kNN'} "
                      f"leaf arithmetic, {cores} threads",
            "agrees_with_gpu": f"{agree}/{n}"}


def run_gts(args):
    import torch
    import torch.distributed as dist

    import gts_b200 as gts

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    rows, qids = workload(args, rank)
    d_rows = torch.from_numpy(rows).to(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = gts.Index.from_device(d_rows.data_ptr(), args.n, args.dim, 2, max_h=args.max_h,
                                stream=stream.cuda_stream)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    del d_rows
    form = {"fast": gts.FORM_FAST, "plain": gts.FORM_PLAIN, "plain-learned": gts.FORM_PLAIN_LEARNED}[args.form]
    learn = None
    rng = args.op == "range"
    if rng and args.form == "plain-learned":
        raise SystemExit("--op range takes --form fast or plain")
    if args.form in ("fast", "plain-learned") and not args.no_learn and not rng:
        # learned radius: 200,000 exact radii from the index itself, trained on
        # the device before the timed region
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        learn = idx.learn_radius(n_train=args.train, k_max=64, epochs=12, seed=args.seed)
        torch.cuda.synchronize()
        learn["train_s"] = time.perf_counter() - t0
        learn["n_train"] = args.train
    Q = args.queries
    # one batch per k (one in all unless --k-mix): device ids and results
    groups = []
    for k, sel in k_groups(args, Q):
        groups.append({"k": k, "sel": sel, "q": torch.from_numpy(np.ascontiguousarray(qids[sel])).to(dev),
                       "kth": torch.empty(len(sel), dtype=torch.int32 if rng else torch.float32, device=dev)})
    k = groups[0]["k"] if len(groups) == 1 else None

    def run_group(g):
        if rng:
            idx.range_device(g["q"].data_ptr(), len(g["sel"]), args.radius, g["kth"].data_ptr(),
                             stream=stream.cuda_stream, form=form)
        else:
            idx.knn_device(g["q"].data_ptr(), len(g["sel"]), g["k"], g["kth"].data_ptr(), form=form,
                           stream=stream.cuda_stream)

    def step():
        for g in groups:
            run_group(g)

    if learn is not None and args.form == "fast" and args.learned_seed != "auto":
        step()   # tunes the configuration for each k, then the seed choice is pinned
        torch.cuda.synchronize()
        for g in groups:
            c = idx.fast_config(g["k"])
            idx.set_fast_config(g["k"], args.learned_seed == "on", c["col_groups"], c["item_blocks"])
    clocks = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
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
    if args.form == "fast":
        idx.filter_timing(reset=True)
    if args.profile:
        torch.cuda.profiler.start()
    launches0 = idx.kernel_launches()
    wall0 = time.time()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    wall1 = time.time()
    launches = idx.kernel_launches() - launches0
    filter_ms, filter_launches = idx.filter_timing() if args.form == "fast" else (0.0, 0)
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
    total_ms = t_start.elapsed_time(t_end)
    per_launch_ms = [a.elapsed_time(b) for a, b in ev]
    if world > 1:
        from gts_b200 import replicas as R
        total_ms = R.max_over_ranks(total_ms, dist, dev)
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * Q * args.steps / (total_ms / 1e3)
    kth_gpu = np.zeros(Q, np.int32 if rng else np.float32)
    for g in groups:
        kth_gpu[g["sel"]] = g["kth"].cpu().numpy()

    # end to end through the host-buffer API: H2D of the query ids from pinned
    # memory and D2H of the k-th distances inside every timed call
    for g in groups:
        g["h_q"] = torch.from_numpy(np.ascontiguousarray(qids[g["sel"]])).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        for g in groups:
            idx.range(g["h_q"], args.radius, form=form) if rng else idx.knn(g["h_q"], g["k"], form=form)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        kth_e2e = [idx.range(g["h_q"], args.radius, form=form) if rng else idx.knn(g["h_q"], g["k"], form=form)
                   for g in groups]
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = R.max_over_ranks(e2e_s, dist, dev)
    e2e = {"value": world * Q * args.steps / e2e_s, "unit": "queries/s",
           "h2d_bytes_per_step": int(sum(g["h_q"].nbytes for g in groups)),
           "d2h_bytes_per_step": int(sum(x.nbytes for x in kth_e2e))}
    for g, x in zip(groups, kth_e2e):
        assert np.array_equal(x, kth_gpu[g["sel"]]), "host-buffer and device-buffer paths disagree"

    peaks = measured_peaks_all()
    d = args.dim
    launch_ms = statistics.mean(per_launch_ms)
    # DRAM traffic of the dominant kernel per launch: the ncu capture's bytes
    # per unit (operand block for the filter, leaf object for the traversal)
    # times the units this run processed per launch
    per_unit = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            per_unit = json.load(f)
    if args.form != "fast":
        # every leaf row and pivot row a query reads, plus its own row and result
        alg_bytes = 4 * d * (stats["objects"] + stats["pivots"]) + sum(
            len(g["sel"]) * (4 * d + (4 if rng else 8 * g["k"])) for g in groups)
        achieved = alg_bytes / (launch_ms / 1e3) / 1e9
        traffic = None
        if "k_search" in per_unit:
            traffic = per_unit["k_search"]["dram_bytes_per_object"] * stats["objects"]
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                    "peak_kind": peaks["kind"], "kernel": "k_search",
                    "alg_bytes_per_launch": alg_bytes,
                    "per_query": {"leaf_objects": stats["objects"] / Q, "pivots": stats["pivots"] / Q,
                                  "exact_rechecks": stats["exact"] / Q}}
    else:
        # tensor pipe: every streamed block is one 128 x 144 x Kp MMA chain for
        # the BF16 high part and one for the low part of the queries
        # timed on the device around every filter launch (CUDA events on the
        # launching stream); one step runs the filter once, plus once per
        # re-answer stage when queries fail
        kp = (d + 63) // 64 * 64
        per_step = max(1, filter_launches // max(1, args.steps))
        flops = stats["blocks"] * 2 * 128 * 144 * kp * 2 / per_step
        kernel_ms = filter_ms / max(1, filter_launches)
        achieved = flops / (kernel_ms / 1e3) / 1e12
        traffic = None
        if "k_fast_tile" in per_unit:
            traffic = per_unit["k_fast_tile"]["dram_bytes_per_block"] * stats["blocks"] / per_step
        streamed = stats["bytes"] / per_step
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"],
                    "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"], "traffic": traffic,
                    "peak_kind": peaks["kind"], "kernel": "k_fast_tile",
                    "kernel_ms_per_launch": kernel_ms, "launches_per_step": per_step,
                    "kernel_share_of_step": filter_ms / total_ms,
                    "mma_flops_per_launch": flops,
                    "streamed_bytes_per_launch": streamed,
                    "streamed_gbs": streamed / (kernel_ms / 1e3) / 1e9,
                    "streamed_hbm_frac": streamed / (kernel_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
                    "per_query": {"blocks": stats["blocks"] / Q, "appended": stats["appended"] / Q,
                                  "exact_rechecks": stats["exact"] / Q,
                                  "fallback_queries": stats["fallback"], "passes": stats["passes"]},
                    "block_pairs_kept": (stats["blocks"] / stats["tested"]) if stats["tested"] else None}
    line = {"metric": "exact range queries/s" if rng else "exact kNN queries/s", "value": value,
            "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64" if args.form != "fast" else "bf16/f32/f64",
            "data": "synthetic (seeded Gaussian mixture; the paper's data sets are absent)",
            "config": config_dict(args, world), "build_s": build_s, "learned_radius": learn,
            "autotune": (({"col_groups": 4, "item_blocks": 16, "tuned": False} if rng
                          else idx.fast_config(k) if k is not None
                          else {str(g["k"]): idx.fast_config(g["k"]) for g in groups})
                         if args.form == "fast" else {"threads_per_query_cta": idx.plain_threads(1 if rng else 0)}),
            "roofline": roofline,
            "e2e": e2e, "gpu_launches": launches, "clocks": clock_summary}
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        line["cpu_baseline"] = cpu_baseline(rows, qids, groups, args.cpu_sample, kth_gpu,
                                            args.radius if rng else None)
    if rank == 0:
        print(json.dumps(line))
    idx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gts", "reference"], default="gts")
    ap.add_argument("--form", choices=["fast", "plain", "plain-learned"], default="fast",
                    help="plain-learned: the plain traversal seeded by the trained radius")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=128)
    ap.add_argument("--queries", type=int, default=10_000)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--op", choices=["knn", "range"], default="knn",
                    help="range: range counts at the --range-quantile distance quantile")
    ap.add_argument("--range-quantile", type=float, default=0.001)
    ap.add_argument("--k-mix", action="store_true",
                    help="k uniform over {1, 8, 32, 64} per query (one batch per k per step)")
    ap.add_argument("--max-h", type=int, default=6)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample", type=int, default=256)
    ap.add_argument("--no-learn", action="store_true",
                    help="fast form without the learned radius (own-block seeds only)")
    ap.add_argument("--train", type=int, default=200_000, help="learned-radius training samples")
    ap.add_argument("--learned-seed", choices=["auto", "on", "off"], default="auto",
                    help="fast form with a trained radius: let the autotuner choose the learned seed, "
                         "or force it on / off (the other tuned settings are kept)")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    return run_gts(args)


if __name__ == "__main__":
    sys.exit(main())
