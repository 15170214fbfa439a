"""B200-native GTS: exact metric similarity search on a GPU pivot tree.

Python host binding over the C ABI of ``libgts_b200.so`` (include/gts_b200.h).
The compute path is the CUDA library; there is no CPU fallback -- importing
works without a GPU, but every index operation needs the built library and a
CUDA device and raises ``GtsError`` otherwise.

The reference entry points are mirrored by name:

=========================  =============================================
reference (Source Code/GTS)  here
=========================  =============================================
``load`` file.cuh:28        :func:`load`
``loadQuery`` file.cuh:112  :func:`load_queries`
``loadUpdate`` update.cuh:43 :func:`load_updates`
``indexConstru`` tree.cuh:332  :func:`indexConstru` / :class:`Index`
``searchIndexKnnV2`` search_v2.cuh:975  :func:`searchIndexKnnV2` / :meth:`Index.knn`
``searchIndexRnnV2`` search_v2.cuh:780  :func:`searchIndexRnnV2` / :meth:`Index.range`
``updateIndexRnn`` update.cuh:449  :func:`updateIndexRnn` / :meth:`Index.update_run`
``saveK`` / ``saveR`` file.cuh:154-199  :func:`saveK` / :func:`saveR`
=========================  =============================================
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["GtsError", "Params", "Index", "load", "load_queries", "load_updates",
           "indexConstru", "searchIndexKnnV2", "searchIndexRnnV2", "updateIndexRnn",
           "saveK", "saveR", "lib_path", "FORM_PLAIN", "FORM_FAST", "FORM_PLAIN_LEARNED"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgts_b200.so")
STR_STRIDE = 109
FORM_PLAIN, FORM_FAST, FORM_PLAIN_LEARNED = 0, 1, 2
RADIUS_MODEL_PARAMS = 128 * 33 + 128 + 128 * 128 + 128 + 128 + 1
_lib = None


def radius_model_grad(X, target, params, norm):
    """(loss, grad) of the radius model on a batch, from the device kernels."""
    X = np.ascontiguousarray(X, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    P = np.ascontiguousarray(params, np.float32)
    nm = np.ascontiguousarray(norm, np.float32)
    g = np.empty(RADIUS_MODEL_PARAMS, np.float32)
    loss = C.c_float()
    _check(_load_lib().gts_radius_model_grad(_fp(X), _fp(t), len(t), _fp(P), _fp(nm), _fp(g),
                                             C.byref(loss)))
    return loss.value, g


class GtsError(RuntimeError):
    """A GTS C-ABI call failed (message from gts_last_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"GTS error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    """Runtime tunables; defaults are the reference's compile-time values
    (tree.cuh:31-35, update.cuh:16)."""
    _fields_ = [("tree_order", C.c_int), ("max_size", C.c_int), ("max_h", C.c_int),
                ("dis_code", C.c_int), ("infi_dis", C.c_int), ("max_in_size", C.c_int),
                ("mem_budget_gb", C.c_double)]

    def __init__(self, tree_order=10, max_size=20, max_h=3, dis_code=100, infi_dis=10000,
                 max_in_size=10, mem_budget_gb=0.0):
        super().__init__(tree_order, max_size, max_h, dis_code, infi_dis, max_in_size,
                         mem_budget_gb)


class _Info(C.Structure):
    _fields_ = [("num", C.c_int), ("dim", C.c_int), ("metric", C.c_int), ("tree_h", C.c_int),
                ("max_node_num", C.c_int), ("tree_order", C.c_int), ("max_size", C.c_int),
                ("device_bytes", C.c_size_t)]


def lib_path() -> str:
    return _LIB_PATH


def _load_lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(
            f"{_LIB_PATH} is not built; run `python -m gts_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(_LIB_PATH)
    lib.gts_last_error.restype = C.c_char_p
    _lib = lib
    return lib


def _check(rc: int):
    if rc != 0:
        raise GtsError(rc, _load_lib().gts_last_error().decode(errors="replace"))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


# --------------------------------------------------------------------- I/O

def load(path: str):
    """Reference text data file -> (dim, num, metric, rows | (strs, lens))."""
    lib = _load_lib()
    dim, num, metric = C.c_int(), C.c_int(), C.c_int()
    rows, strs, lens = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(lib.gts_load(path.encode(), C.byref(dim), C.byref(num), C.byref(metric),
                        C.byref(rows), C.byref(strs), C.byref(lens)))
    n, d, m = num.value, dim.value, metric.value
    try:
        if m == 6:
            s = np.ctypeslib.as_array(C.cast(strs, C.POINTER(C.c_uint8)), (n, STR_STRIDE)).copy()
            ln = np.ctypeslib.as_array(C.cast(lens, C.POINTER(C.c_int)), (n,)).copy()
            return d, n, m, (s, ln)
        r = np.ctypeslib.as_array(C.cast(rows, C.POINTER(C.c_float)), (n, d)).copy()
        return d, n, m, r
    finally:
        for p in (rows, strs, lens):
            if p.value:
                lib.gts_free_host(p)


def load_queries(path: str) -> np.ndarray:
    lib = _load_lib()
    q, n = C.c_void_p(), C.c_int()
    _check(lib.gts_load_queries(path.encode(), C.byref(q), C.byref(n)))
    try:
        return np.ctypeslib.as_array(C.cast(q, C.POINTER(C.c_int)), (n.value,)).copy() \
            if n.value else np.zeros(0, np.int32)
    finally:
        lib.gts_free_host(q)


def load_updates(path: str):
    lib = _load_lib()
    f, i, n = C.c_void_p(), C.c_void_p(), C.c_int()
    _check(lib.gts_load_updates(path.encode(), C.byref(f), C.byref(i), C.byref(n)))
    try:
        if n.value == 0:
            return np.zeros(0, np.int32), np.zeros(0, np.int32)
        return (np.ctypeslib.as_array(C.cast(f, C.POINTER(C.c_int)), (n.value,)).copy(),
                np.ctypeslib.as_array(C.cast(i, C.POINTER(C.c_int)), (n.value,)).copy())
    finally:
        lib.gts_free_host(f)
        lib.gts_free_host(i)


def saveK(path_ids: str, path_dis: str, ids: np.ndarray, dists: np.ndarray) -> None:
    """saveK layout (file.cuh:154-176): one line of k ids / k distances per query."""
    with open(path_ids, "w") as fr, open(path_dis, "w") as fd:
        for row_i, row_d in zip(ids, dists):
            fr.write("".join(f"{int(v)} " for v in row_i) + "\n")
            fd.write("".join(f"{float(v):f} " for v in row_d) + "\n")


def saveR(path_ids: str, path_dis: str, ids, dists, counts, offsets) -> None:
    """saveR layout (file.cuh:178-199): appended, one line per query."""
    with open(path_ids, "a") as fr, open(path_dis, "a") as fd:
        for c, o in zip(counts, offsets):
            fr.write("".join(f"{int(v)} " for v in ids[o:o + c]) + "\n")
            fd.write("".join(f"{float(v):f} " for v in dists[o:o + c]) + "\n")


# --------------------------------------------------------------------- index

class Index:
    """A GTS pivot tree built and searched on the current CUDA device."""

    def __init__(self, rows=None, metric: int = 2, strs=None, lens=None,
                 params: Params | None = None, **param_kw):
        lib = _load_lib()
        self._lib = lib
        self.params = params if params is not None else Params(**param_kw)
        self._h = C.c_void_p()
        if metric == 6:
            strs = np.ascontiguousarray(strs, dtype=np.uint8)
            lens = np.ascontiguousarray(lens, dtype=np.int32)
            if strs.ndim != 2 or strs.shape[1] != STR_STRIDE:
                raise ValueError(f"strs must be (num, {STR_STRIDE}) bytes")
            _check(lib.gts_index_build(1, len(lens), 6, None, strs.ctypes.data_as(C.c_char_p),
                                       _ip(lens), C.byref(self.params), C.byref(self._h)))
        else:
            rows = np.ascontiguousarray(rows, dtype=np.float32)
            if rows.ndim != 2:
                raise ValueError("rows must be (num, dim)")
            _check(lib.gts_index_build(rows.shape[1], rows.shape[0], metric, _fp(rows), None, None,
                                       C.byref(self.params), C.byref(self._h)))
        self.metric = metric

    @classmethod
    def from_device(cls, d_rows_ptr: int, num: int, dim: int, metric: int = 2,
                    params: Params | None = None, stream: int = 0, **param_kw):
        self = cls.__new__(cls)
        self._lib = _load_lib()
        self.params = params if params is not None else Params(**param_kw)
        self._h = C.c_void_p()
        _check(self._lib.gts_index_build_device(dim, num, metric, C.c_void_p(d_rows_ptr), None, None,
                                                C.byref(self.params), C.c_void_p(stream),
                                                C.byref(self._h)))
        self.metric = metric
        return self

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.gts_index_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def info(self) -> dict:
        i = _Info()
        _check(self._lib.gts_index_info_get(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in _Info._fields_}

    def export(self) -> dict:
        inf = self.info
        n, m = inf["num"], inf["max_node_num"]
        out = {"id_list": np.empty(n, np.int32), "pid": np.empty(m, np.int32),
               "min_dis": np.empty(m, np.float32), "size": np.empty(m, np.int32),
               "lid": np.empty(m, np.int32), "is_leaf": np.empty(m, np.int32),
               "exists": np.empty(m, np.int32)}
        _check(self._lib.gts_index_export(self._h, _ip(out["id_list"]), _ip(out["pid"]),
                                          _fp(out["min_dis"]), _ip(out["size"]), _ip(out["lid"]),
                                          _ip(out["is_leaf"]), _ip(out["exists"])))
        out["tree_h"] = inf["tree_h"]
        return out

    def prepare(self, form: int = FORM_FAST, stream: int = 0) -> bool:
        """Build the structures `form` needs beyond the tree now (the fast
        form's filter records); True when the index holds them afterwards."""
        done = C.c_int()
        _check(self._lib.gts_index_prepare(self._h, int(form), C.c_void_p(stream), C.byref(done)))
        return bool(done.value)

    def set_stream(self, stream: int):
        _check(self._lib.gts_index_set_stream(self._h, C.c_void_p(stream)))

    def search_stats(self) -> dict:
        """Work counters of the last search: leaf objects read, pivots
        evaluated, exact recomputations, queries finished."""
        out = (C.c_ulonglong * 8)()
        _check(self._lib.gts_search_stats(self._h, out))
        return {"objects": out[0], "pivots": out[1], "exact": out[2], "queries": out[3],
                "fallback": out[4], "appended": out[5], "passes": out[6],
                # fast form: [0] counts operand blocks and [1] their bytes;
                # [7] the (query tile, block) pairs the block bound tested
                "blocks": out[0], "bytes": out[1], "tested": out[7]}

    def filter_timing(self, reset: bool = False):
        """(milliseconds, launches) of the fast form's filter kernel since the
        last reset, from CUDA events around each launch; reset=True zeroes
        the totals and turns the timing on."""
        ms = C.c_double()
        n = C.c_longlong()
        _check(self._lib.gts_filter_timing(self._h, 1 if reset else 0, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def fast_config(self, k: int) -> dict:
        """The autotuned (or default) fast-form configuration for k."""
        v = [C.c_int() for _ in range(5)]
        _check(self._lib.gts_fast_config(self._h, k, *[C.byref(x) for x in v]))
        return {"tuned": bool(v[0].value), "learned_seed": bool(v[1].value), "col_groups": v[2].value,
                "item_blocks": v[3].value, "streamed": v[4].value == 1, "by_block": v[4].value == 2}

    def fast_seeds(self, qids, k: int) -> np.ndarray:
        """The fast form's starting bound on each query's squared k-th
        distance (made with the filter records; see gts_fast_seeds)."""
        q = np.ascontiguousarray(qids, dtype=np.int32)
        out = np.empty(len(q), np.float32)
        _check(self._lib.gts_fast_seeds(self._h, _ip(q), len(q), k, _fp(out)))
        return out

    def fast_graphs(self, on=None) -> int:
        """Turn the captured filter graph on/off (None: leave it); returns the
        number of graph replays so far."""
        n = C.c_longlong()
        _check(self._lib.gts_fast_graphs(self._h, -1 if on is None else int(bool(on)), C.byref(n)))
        return n.value

    def set_fast_config(self, k: int, learned_seed: bool, col_groups: int, item_blocks: int = 16,
                        streamed: bool = False, by_block: bool = False):
        """Pin the fast-form configuration for k instead of tuning it
        (by_block: the block-stationary filter; col_groups and item_blocks
        are then unused)."""
        _check(self._lib.gts_fast_config_set(self._h, k, int(bool(learned_seed)), col_groups, item_blocks,
                                             2 if by_block else int(bool(streamed))))

    def fast_range_variant(self, variant=None) -> int:
        """Filter of the fast range counts: 0 the block-stationary one where
        it fits, 1 the tile one (default); None leaves it.  Returns it."""
        cur = C.c_int()
        _check(self._lib.gts_fast_range_variant(self._h, -1 if variant is None else int(variant), C.byref(cur)))
        return cur.value

    def fast_autotune_reset(self):
        _check(self._lib.gts_fast_autotune_reset(self._h))

    def plain_threads(self, mode: int = 0) -> int:
        """Threads per query CTA of the plain traversal for a search mode
        (0 kNN, 1 range count, 2 range ids); 0 = not tuned yet."""
        n = C.c_int()
        _check(self._lib.gts_plain_threads(self._h, mode, C.byref(n)))
        return n.value

    def set_plain_threads(self, mode: int, threads: int):
        """Pin the plain traversal's threads per query CTA (128/256/512, 0 = tune)."""
        _check(self._lib.gts_plain_threads_set(self._h, mode, threads))

    def plain_split(self, objects: int | None = None) -> int:
        """Set the range traversal's hand-over threshold (objects verified by
        one query in one CTA; 0 = off; None leaves it); returns the number of
        (query, node) items handed over so far."""
        n = C.c_longlong()
        _check(self._lib.gts_plain_split(self._h, -1 if objects is None else int(objects), C.byref(n)))
        return n.value

    def kernel_launches(self) -> int:
        """Kernels this library launched for searches on this handle so far."""
        n = C.c_longlong()
        _check(self._lib.gts_kernel_launches(self._h, C.byref(n)))
        return n.value

    def knn(self, qids, k: int, form: int = FORM_PLAIN, return_ids: bool = False):
        q = np.ascontiguousarray(qids, dtype=np.int32)
        kth = np.empty(len(q), np.float32)
        ids = np.empty((len(q), k), np.int32) if return_ids else None
        dis = np.empty((len(q), k), np.float32) if return_ids else None
        _check(self._lib.gts_knn(self._h, _ip(q), len(q), k, form, _fp(kth),
                                 _ip(ids) if return_ids else None,
                                 _fp(dis) if return_ids else None))
        return (kth, ids, dis) if return_ids else kth

    def knn_device(self, d_qids: int, qnum: int, k: int, d_kth: int, d_ids: int = 0,
                   d_dists: int = 0, form: int = FORM_PLAIN, stream: int = 0):
        _check(self._lib.gts_knn_device(self._h, C.c_void_p(d_qids), qnum, k, form,
                                        C.c_void_p(d_kth), C.c_void_p(d_ids or None),
                                        C.c_void_p(d_dists or None), C.c_void_p(stream)))

    def _query_data(self, queries):
        if self.metric == 6:
            strs, lens = queries
            strs = np.ascontiguousarray(strs, dtype=np.uint8)
            lens = np.ascontiguousarray(lens, dtype=np.int32)
            if strs.ndim != 2 or strs.shape[1] != STR_STRIDE:
                raise ValueError(f"query strings must be (n, {STR_STRIDE}) bytes")
            return None, strs, lens, len(lens)
        rows = np.ascontiguousarray(queries, dtype=np.float32)
        if rows.ndim != 2:
            raise ValueError("query rows must be (n, dim)")
        return rows, None, None, rows.shape[0]

    def knn_rows(self, queries, k: int, return_ids: bool = False):
        """kNN of queries given as data (rows, or (strs, lens) for metric 6),
        not object ids: no self match."""
        rows, strs, lens, n = self._query_data(queries)
        kth = np.empty(n, np.float32)
        ids = np.empty((n, k), np.int32) if return_ids else None
        dis = np.empty((n, k), np.float32) if return_ids else None
        _check(self._lib.gts_knn_rows(self._h, _fp(rows) if rows is not None else None,
                                      strs.ctypes.data_as(C.c_char_p) if strs is not None else None,
                                      _ip(lens) if lens is not None else None, n, k, _fp(kth),
                                      _ip(ids) if return_ids else None, _fp(dis) if return_ids else None))
        return (kth, ids, dis) if return_ids else kth

    def range_rows(self, queries, r: float) -> np.ndarray:
        """Range counts of queries given as data (see knn_rows)."""
        rows, strs, lens, n = self._query_data(queries)
        out = np.empty(n, np.int32)
        _check(self._lib.gts_range_rows(self._h, _fp(rows) if rows is not None else None,
                                        strs.ctypes.data_as(C.c_char_p) if strs is not None else None,
                                        _ip(lens) if lens is not None else None, n, C.c_float(r), _ip(out)))
        return out

    def range(self, qids, r: float, form: int = FORM_PLAIN) -> np.ndarray:
        """Count of objects within r of each query (itself included);
        form=FORM_FAST runs the tensor-core filter (L2, dim <= 128)."""
        q = np.ascontiguousarray(qids, dtype=np.int32)
        out = np.empty(len(q), np.int32)
        if form == FORM_PLAIN:
            _check(self._lib.gts_range(self._h, _ip(q), len(q), C.c_float(r), _ip(out)))
        else:
            _check(self._lib.gts_range_form(self._h, _ip(q), len(q), C.c_float(r), int(form), _ip(out)))
        return out

    def range_device(self, d_qids: int, qnum: int, r: float, d_counts: int, stream: int = 0,
                     form: int = FORM_PLAIN):
        if form == FORM_PLAIN:
            _check(self._lib.gts_range_device(self._h, C.c_void_p(d_qids), qnum, C.c_float(r),
                                              C.c_void_p(d_counts), C.c_void_p(stream)))
        else:
            _check(self._lib.gts_range_form_device(self._h, C.c_void_p(d_qids), qnum, C.c_float(r), int(form),
                                                   C.c_void_p(d_counts), C.c_void_p(stream)))

    def range_ids(self, qids, r: float, capacity: int | None = None):
        """-> (counts, offsets, ids, dists); each query's hits in (distance, id) order."""
        q = np.ascontiguousarray(qids, dtype=np.int32)
        counts = np.empty(len(q), np.int32)
        offs = np.empty(len(q), np.int32)
        if capacity is None:
            capacity = int(self.range(q, r).sum())
        ids = np.empty(max(capacity, 1), np.int32)
        dis = np.empty(max(capacity, 1), np.float32)
        _check(self._lib.gts_range_ids(self._h, _ip(q), len(q), C.c_float(r), _ip(counts),
                                       _ip(offs), _ip(ids), _fp(dis), C.c_size_t(capacity)))
        tot = int(counts.sum())
        return counts, offs, ids[:tot], dis[:tot]

    def learn_radius(self, n_train: int = 200_000, k_max: int = 64, epochs: int = 12,
                     seed: int = 0) -> dict:
        """Train the learned kNN radius (GTS_FORM_FAST then starts from it)."""
        rmse, widen = C.c_float(), C.c_float()
        _check(self._lib.gts_learn_radius(self._h, n_train, k_max, epochs, C.c_uint(seed),
                                          C.byref(rmse), C.byref(widen)))
        return {"val_rmse_log": rmse.value, "widen": widen.value}

    def radius_model(self) -> dict:
        P = np.empty(RADIUS_MODEL_PARAMS, np.float32)
        norm = np.empty(66, np.float32)
        extra = np.empty(3, np.float32)
        _check(self._lib.gts_radius_model_params(self._h, _fp(P), _fp(norm), _fp(extra)))
        return {"params": P, "norm": norm, "ymu": float(extra[0]), "ysig": float(extra[1]),
                "widen": float(extra[2])}

    def update_run_rows(self, flags, ids, new_rows, r: float):
        """The stream with inserts that bring new rows (flag 0 with id j
        inserts new_rows[j]) -> (counts per query op, search s, update s)."""
        f = np.ascontiguousarray(flags, dtype=np.int32)
        i = np.ascontiguousarray(ids, dtype=np.int32)
        nr = np.ascontiguousarray(new_rows, dtype=np.float32)
        out = np.empty(max(1, int((f == 2).sum())), np.int32)
        nq = C.c_int()
        ts, tu = C.c_double(), C.c_double()
        _check(self._lib.gts_update_run_rows(self._h, _ip(f), _ip(i), len(f), _fp(nr) if len(nr) else None, len(nr),
                                             C.c_float(r), _ip(out), C.byref(nq), C.byref(ts), C.byref(tu)))
        return out[:nq.value], ts.value, tu.value

    def update_run(self, flags, ids, r: float):
        """-> (counts per query op, search seconds, update seconds)."""
        f = np.ascontiguousarray(flags, dtype=np.int32)
        i = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.empty(max(1, int((f == 2).sum())), np.int32)
        nq = C.c_int()
        ts, tu = C.c_double(), C.c_double()
        _check(self._lib.gts_update_run(self._h, _ip(f), _ip(i), len(f), C.c_float(r), _ip(out),
                                        C.byref(nq), C.byref(ts), C.byref(tu)))
        return out[:nq.value], ts.value, tu.value


def update_plan(num: int, flags, ids, max_in_size: int = 10, n_new: int = 0) -> dict:
    """The host pass of the stream update (updateIndexRnn's id bookkeeping,
    update.cuh:473-623) with no device work: per query op its data row, its
    operation index and whether the cache list held entries; per entry (the
    num data rows, then one copy per insert) the row it copies and its
    (tree_from, tree_to, cache_from, cache_to) operation intervals; the data
    rows after the last compaction.  n_new > 0: a flag-0 op with id j brings
    new row j (object num + j) instead of copying a physical row."""
    f = np.ascontiguousarray(flags, dtype=np.int32)
    i = np.ascontiguousarray(ids, dtype=np.int32)
    nq_cap = max(1, int((f == 2).sum()))
    ne_cap = num + int((f == 0).sum()) + n_new
    q_obj, q_time, q_cache = (np.empty(nq_cap, np.int32) for _ in range(3))
    src = np.empty(ne_cap, np.int32)
    life = np.empty((ne_cap, 4), np.int32)
    final = np.empty(max(1, ne_cap), np.int32)
    nq, ne, nf = C.c_int(), C.c_int(), C.c_int()
    _check(_load_lib().gts_update_plan(num, _ip(f), _ip(i), len(f), max_in_size, n_new, _ip(q_obj), _ip(q_time),
                                       _ip(q_cache), C.byref(nq), _ip(src), _ip(life), C.byref(ne),
                                       _ip(final), C.byref(nf)))
    return {"q_obj": q_obj[:nq.value], "q_time": q_time[:nq.value], "q_cache": q_cache[:nq.value].astype(bool),
            "ent_src": src[:ne.value], "ent_life": life[:ne.value], "final_rows": final[:nf.value]}


# ------------------------------------------------- reference-named wrappers

def indexConstru(rows=None, metric: int = 2, strs=None, lens=None, **params) -> Index:
    """indexConstru (tree.cuh:332): build the index."""
    return Index(rows, metric, strs, lens, **params)


def searchIndexKnnV2(index: Index, qids, k: int) -> np.ndarray:
    """searchIndexKnnV2 (search_v2.cuh:975): -> res_dis, the k-th distance per query."""
    return index.knn(qids, k)


def searchIndexRnnV2(index: Index, qids, r: float) -> np.ndarray:
    """searchIndexRnnV2 (search_v2.cuh:780): -> res, the result count per query."""
    return index.range(qids, r)


def _write_fcost(fcost, values, fmt):
    """The per-query line the reference's v1 search appends to its cost file
    (search.cuh:857-861, 1043-1047): values separated by single spaces."""
    if fcost is None:
        return
    text = "".join((fmt % v) + " " for v in values)
    if hasattr(fcost, "write"):
        fcost.write(text)
        fcost.flush()
    else:
        with open(fcost, "a") as f:
            f.write(text)


def searchIndexRnn(index: Index, qids, r: float, fcost=None):
    """searchIndexRnn, the v1 multi-query range search (search.cuh:749-889):
    -> (qresult_count, qresult_count_prefix, result_id, result_dis), the hits
    of query i at result_id[prefix[i] : prefix[i] + count[i]].  The same
    traversal as the v2 entry point answers it (exact on every tree shape);
    each query's hits come in (distance, id) order, where the reference keeps
    its leaf-pair order (the same sets).  fcost (an open file or a path, or
    None) receives the counts as the reference writes them."""
    counts, offs, ids, dis = index.range_ids(qids, r)
    _write_fcost(fcost, counts, "%d")
    return counts, offs, ids, dis


def searchIndexKnn(index: Index, qids, k: int, fcost=None):
    """searchIndexKnn, the v1 multi-query kNN search (search.cuh:891-1081):
    -> (result_id, result_dis), k entries per query at [i*k : (i+1)*k] in
    ascending distance, ties by id (the reference breaks ties by its
    candidate order).  Slots past the number of objects hold id -1 and
    distance INFI_DIS.  fcost receives the k-th distances as the reference
    writes them (%f)."""
    kth, ids, dis = index.knn(qids, k, return_ids=True)
    _write_fcost(fcost, kth, "%f")
    return ids.reshape(-1), dis.reshape(-1)


def updateIndexRnn(index: Index, flags, ids, r: float) -> np.ndarray:
    """updateIndexRnn (update.cuh:449): -> the result count of every query op."""
    return index.update_run(flags, ids, r)[0]
