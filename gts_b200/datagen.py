"""Seeded synthetic workloads in the shapes GTS is benchmarked on.

The GTS paper's datasets (Words, T-Loc, Vector, DNA, Color; reference
README.md:119-131) are not available here, so these generators stand in for
them at the same shapes and value distributions:

* ``gmm_rows``       -- Gaussian-mixture float32 vectors (Vector-like; L2)
* ``word_strings``   -- lowercase words, log-normal lengths, Zipf letters
                        (Words-like; edit distance)
* ``hotspot_points`` -- 2-D points, 70% in Gaussian hotspots (T-Loc-like; L1)
* ``update_stream``  -- insert / delete / query operations whose ids are valid
                        under the reference's id semantics (update.cuh:449-638)

Writers produce the reference's text formats (file.cuh:28-152,
update.cuh:43-95) and a binary form (int32 dim, num, metric; then rows).
"""
from __future__ import annotations

import numpy as np

STR_STRIDE = 109  # row stride of string objects (file.cuh:15)

METRIC_LINF, METRIC_L1, METRIC_L2, METRIC_ANGLE, METRIC_EDIT = 0, 1, 2, 5, 6


def gmm_rows(n: int, dim: int, n_comp: int, sigma: float, seed: int) -> np.ndarray:
    """n x dim float32 rows: centres ~ N(0, 1), per-cluster isotropic sigma."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((n_comp, dim)).astype(np.float32)
    comp = rng.integers(0, n_comp, size=n)
    out = np.empty((n, dim), dtype=np.float32)
    step = 1 << 18
    for s in range(0, n, step):
        e = min(n, s + step)
        out[s:e] = centres[comp[s:e]] + sigma * rng.standard_normal((e - s, dim), dtype=np.float32)
    return out


def word_strings(n: int, seed: int, median: float = 8.0, max_len: int = 34,
                 zipf_s: float = 1.1, log_sigma: float = 0.5):
    """n lowercase strings: (n x STR_STRIDE uint8 buffer, int32 lengths).

    Lengths follow a log-normal with the given median clipped to
    [1, max_len]; letters are Zipf(zipf_s)-distributed over a..z."""
    rng = np.random.default_rng(seed)
    lens = np.exp(np.log(median) + log_sigma * rng.standard_normal(n))
    lens = np.clip(np.rint(lens), 1, max_len).astype(np.int32)
    ranks = np.arange(1, 27, dtype=np.float64)
    p = ranks ** (-zipf_s)
    p /= p.sum()
    letters = rng.choice(np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", dtype=np.uint8),
                         size=(n, max_len), p=p)
    buf = np.zeros((n, STR_STRIDE), dtype=np.uint8)
    mask = np.arange(max_len)[None, :] < lens[:, None]
    buf[:, :max_len] = np.where(mask, letters, 0)
    return buf, lens


def hotspot_points(n: int, seed: int, n_hot: int = 500, frac_hot: float = 0.7,
                   sigma: float = 0.005) -> np.ndarray:
    """n x 2 float32 points: frac_hot in Gaussian hotspots, the rest uniform."""
    rng = np.random.default_rng(seed)
    hot = rng.random((n_hot, 2))
    n_h = int(round(n * frac_hot))
    pts = np.empty((n, 2), dtype=np.float64)
    pts[:n_h] = hot[rng.integers(0, n_hot, size=n_h)] + sigma * rng.standard_normal((n_h, 2))
    pts[n_h:] = rng.random((n - n_h, 2))
    rng.shuffle(pts, axis=0)
    return pts.astype(np.float32)


def query_ids(n: int, q: int, seed: int) -> np.ndarray:
    """q query ids drawn uniformly (without replacement when q <= n)."""
    rng = np.random.default_rng(seed)
    return rng.choice(n, size=q, replace=q > n).astype(np.int32)


def _levenshtein(a: bytes, b: bytes) -> int:
    if not a:
        return len(b)
    if not b:
        return len(a)
    prev = list(range(len(b) + 1))
    for i, ca in enumerate(a, 1):
        cur = [i] + [0] * len(b)
        for j, cb in enumerate(b, 1):
            cur[j] = min(prev[j] + 1, cur[j - 1] + 1, prev[j - 1] + (ca != cb))
        prev = cur
    return prev[-1]


def quantile_radius(metric: int, q: float, n_pairs: int, seed: int, rows=None,
                    strs=None, lens=None) -> float:
    """The q-quantile of n_pairs seeded random pair distances (float64 math)."""
    rng = np.random.default_rng(seed)
    n = len(rows) if rows is not None else len(lens)
    a = rng.integers(0, n, size=n_pairs)
    b = rng.integers(0, n, size=n_pairs)
    if metric == METRIC_EDIT:
        d = np.array([_levenshtein(bytes(strs[i, :lens[i]]), bytes(strs[j, :lens[j]]))
                      for i, j in zip(a, b)], dtype=np.float64)
    else:
        d = np.empty(n_pairs)
        step = 1 << 16
        for s in range(0, n_pairs, step):
            e = min(n_pairs, s + step)
            diff = rows[a[s:e]].astype(np.float64) - rows[b[s:e]].astype(np.float64)
            if metric == METRIC_L2:
                d[s:e] = np.sqrt((diff * diff).sum(1))
            elif metric == METRIC_L1:
                d[s:e] = np.abs(diff).sum(1)
            elif metric == METRIC_LINF:
                d[s:e] = np.abs(diff).max(1)
            else:
                x = rows[a[s:e]].astype(np.float64)
                y = rows[b[s:e]].astype(np.float64)
                c = (x * y).sum(1) / np.sqrt((x * x).sum(1) * (y * y).sum(1))
                d[s:e] = np.degrees(np.arccos(np.clip(c, -1, 1)))
    return float(np.quantile(d, q))


def update_stream(n: int, n_ops: int, seed: int, max_in_size: int = 10,
                  p_insert: float = 0.45, p_delete: float = 0.45):
    """(flags, ids) for the stream-update path with ids valid at every step.

    The reference's id semantics (update.cuh:449-638): an insert names a
    physical row of the current data array and appends a copy of it to the
    cache list; a delete names a logical id (live tree rows in physical
    order, then the cache list); a query names a physical row.  After
    max_in_size inserts the data is compacted and rebuilt.

    Between two compactions only a handful of rows die (about as many
    deletes as the max_in_size inserts), so the rows deleted since the last
    compaction are a short sorted list: the (u+1)-th live row is u shifted
    past every dead row at or before it.  O(deletes per compaction) per op,
    nothing per compaction, for streams of millions of operations."""
    import bisect
    rng = np.random.default_rng(seed)
    flags = np.empty(n_ops, dtype=np.int32)
    ids = np.empty(n_ops, dtype=np.int32)
    tree_size, ndel, in_size = n, 0, 0
    dead = []          # physical rows deleted since the last compaction, ascending
    dead_set = set()
    u = rng.random(n_ops)
    for i in range(n_ops):
        live = tree_size - ndel + in_size
        if u[i] < p_insert:
            flags[i], ids[i] = 0, rng.integers(0, tree_size)
            in_size += 1
            if in_size == max_in_size:
                tree_size = tree_size - ndel + in_size
                ndel, in_size = 0, 0
                dead, dead_set = [], set()
        elif u[i] < p_insert + p_delete and live > 1:
            lid = int(rng.integers(0, live))
            flags[i], ids[i] = 1, lid
            if lid < tree_size - ndel:
                phys = lid
                for d in dead:
                    if d <= phys:
                        phys += 1
                    else:
                        break
                bisect.insort(dead, phys)
                dead_set.add(phys)
                ndel += 1
            else:
                in_size -= 1
        else:
            # queries name a live physical row, so the query object itself is
            # always a hit (the reference allocates its result arrays by the
            # hit count and stops on a zero-byte managed allocation)
            q = int(rng.integers(0, tree_size))
            while q in dead_set:
                q = int(rng.integers(0, tree_size))
            flags[i], ids[i] = 2, q
    return flags, ids


def update_stream_new_rows(n: int, n_ops: int, seed: int, max_in_size: int = 10, **kw):
    """update_stream whose inserts bring new rows: (flags, ids) with every
    flag-0 id replaced by the running insert number 0, 1, 2, ... (the row of
    the new-row array it inserts); deletes and queries as update_stream's
    (their validity does not depend on the inserted rows' contents)."""
    flags, ids = update_stream(n, n_ops, seed, max_in_size, **kw)
    ins = flags == 0
    ids = ids.copy()
    ids[ins] = np.arange(int(ins.sum()), dtype=np.int32)
    return flags, ids


# --------------------------------------------------------------------------
# writers / readers
# --------------------------------------------------------------------------

def write_data_text(path: str, metric: int, rows=None, strs=None, lens=None) -> None:
    """Reference text format: header 'dim num metric', then one object per line."""
    with open(path, "w") as f:
        if metric == METRIC_EDIT:
            f.write(f"1 {len(lens)} {metric}\n")
            for i in range(len(lens)):
                f.write(bytes(strs[i, :lens[i]]).decode("ascii"))
                f.write("\n")
        else:
            n, dim = rows.shape
            f.write(f"{dim} {n} {metric}\n")
            for i in range(n):
                f.write(" ".join(f"{v:.6f}" for v in rows[i]))
                f.write("\n")


def write_data_bin(path: str, metric: int, rows: np.ndarray) -> None:
    with open(path, "wb") as f:
        np.array([rows.shape[1], rows.shape[0], metric], dtype=np.int32).tofile(f)
        np.ascontiguousarray(rows, dtype=np.float32).tofile(f)


def write_queries(path: str, qids) -> None:
    with open(path, "w") as f:
        f.write(f"{len(qids)}\n")
        for q in qids:
            f.write(f"{int(q)}\n")


def write_updates(path: str, flags, ids) -> None:
    with open(path, "w") as f:
        f.write(f"{len(flags)}\n")
        for fl, i in zip(flags, ids):
            f.write(f"{int(fl)} {int(i)}\n")


def read_text_rows(path: str):
    """Parse a reference text data file -> (metric, rows | (strs, lens))."""
    with open(path, "rb") as f:
        head = f.readline().split()
        dim, num, metric = int(head[0]), int(head[1]), int(head[2])
        if metric == METRIC_EDIT:
            strs = np.zeros((num, STR_STRIDE), dtype=np.uint8)
            lens = np.zeros(num, dtype=np.int32)
            for i in range(num):
                line = f.readline().rstrip(b"\n")
                strs[i, :len(line)] = np.frombuffer(line[:STR_STRIDE], dtype=np.uint8)
                lens[i] = len(line)
            return metric, (strs, lens)
        rows = np.loadtxt(f, dtype=np.float32, max_rows=num, ndmin=2)
        return metric, rows.reshape(num, dim)
