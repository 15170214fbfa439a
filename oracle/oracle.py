"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

STR_STRIDE = 109


class _Data(C.Structure):
    _fields_ = [("dim", C.c_int), ("num", C.c_int), ("metric", C.c_int),
                ("rows", C.c_void_p), ("strs", C.c_void_p), ("lens", C.c_void_p)]


class _Params(C.Structure):
    _fields_ = [("order", C.c_int), ("max_size", C.c_int), ("max_h", C.c_int),
                ("dis_code", C.c_int), ("infi_dis", C.c_int)]


class _Tree(C.Structure):
    _fields_ = [("max_node_num", C.c_int), ("tree_h", C.c_int), ("start_idx", C.c_int),
                ("id_list", C.POINTER(C.c_int)), ("pid", C.POINTER(C.c_int)),
                ("min_dis", C.POINTER(C.c_float)), ("size", C.POINTER(C.c_int)),
                ("lid", C.POINTER(C.c_int)), ("is_leaf", C.POINTER(C.c_int)),
                ("exists", C.POINTER(C.c_int))]


def build_lib() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_lib()
        _lib = C.CDLL(_LIB_PATH)
        _lib.orc_dist.restype = C.c_double
    return _lib


class Dataset:
    """Host dataset in the reference layout, kept alive for the C calls."""

    def __init__(self, metric: int, rows=None, strs=None, lens=None):
        self.metric = metric
        if metric == 6:
            self.strs = np.ascontiguousarray(strs, dtype=np.uint8)
            self.lens = np.ascontiguousarray(lens, dtype=np.int32)
            self.rows = None
            self.num, self.dim = len(self.lens), 1
        else:
            self.rows = np.ascontiguousarray(rows, dtype=np.float32)
            self.strs = self.lens = None
            self.num, self.dim = self.rows.shape
        self._c = _Data(self.dim, self.num, metric,
                        self.rows.ctypes.data if self.rows is not None else None,
                        self.strs.ctypes.data if self.strs is not None else None,
                        self.lens.ctypes.data if self.lens is not None else None)

    @property
    def ref(self):
        return C.byref(self._c)


def params(order=10, max_size=20, max_h=3, dis_code=100, infi_dis=10000):
    return _Params(order, max_size, max_h, dis_code, infi_dis)


def dist(ds: Dataset, a: int, b: int, acc64: bool) -> float:
    return lib().orc_dist(ds.ref, a, b, 1 if acc64 else 0)


class Tree:
    """Result of the restated index construction (tree.cuh:332-393)."""

    def __init__(self, ds: Dataset, p: _Params):
        self._t = _Tree()
        rc = lib().orc_build(ds.ref, C.byref(p), C.byref(self._t))
        if rc != 0:
            raise RuntimeError(f"orc_build failed: {rc}")
        t = self._t
        m, n = t.max_node_num, ds.num
        self.max_node_num, self.tree_h, self.start_idx = m, t.tree_h, t.start_idx
        self.id_list = np.ctypeslib.as_array(t.id_list, (n,)).copy()
        self.pid = np.ctypeslib.as_array(t.pid, (m,)).copy()
        self.min_dis = np.ctypeslib.as_array(t.min_dis, (m,)).copy()
        self.size = np.ctypeslib.as_array(t.size, (m,)).copy()
        self.lid = np.ctypeslib.as_array(t.lid, (m,)).copy()
        self.is_leaf = np.ctypeslib.as_array(t.is_leaf, (m,)).copy()
        self.exists = np.ctypeslib.as_array(t.exists, (m,)).copy()

    def __del__(self):
        try:
            lib().orc_tree_free(C.byref(self._t))
        except Exception:
            pass


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def knn_v2(ds, p, tree: Tree, qids, k: int) -> np.ndarray:
    q = np.ascontiguousarray(qids, dtype=np.int32)
    out = np.empty(len(q), dtype=np.float32)
    rc = lib().orc_knn_v2(ds.ref, C.byref(p), C.byref(tree._t), _iptr(q), len(q), k, _fptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_knn_v2 failed: {rc}")
    return out


def range_v2(ds, p, tree: Tree, qids, r: float) -> np.ndarray:
    q = np.ascontiguousarray(qids, dtype=np.int32)
    out = np.empty(len(q), dtype=np.int32)
    lib().orc_range_v2(ds.ref, C.byref(p), C.byref(tree._t), _iptr(q), len(q),
                       C.c_float(r), _iptr(out))
    return out


def knn_brute(ds, qids, k: int, infi_dis: int = 10000, nthreads: int = 0):
    """-> (kth float32[Q], ids int32[Q,k], dists float32[Q,k]), ties by id."""
    q = np.ascontiguousarray(qids, dtype=np.int32)
    kth = np.empty(len(q), dtype=np.float32)
    ids = np.empty((len(q), k), dtype=np.int32)
    dis = np.empty((len(q), k), dtype=np.float32)
    lib().orc_knn_brute(ds.ref, _iptr(q), len(q), k, infi_dis, _fptr(kth), _iptr(ids),
                        _fptr(dis), nthreads)
    return kth, ids, dis


def range_brute(ds, qids, r: float, nthreads: int = 0) -> np.ndarray:
    q = np.ascontiguousarray(qids, dtype=np.int32)
    out = np.empty(len(q), dtype=np.int32)
    lib().orc_range_brute(ds.ref, _iptr(q), len(q), C.c_float(r), _iptr(out), nthreads)
    return out


def update_run_rows(ds, max_in_size: int, flags, ids, new_rows, r: float) -> np.ndarray:
    """Counts per query op of a stream whose inserts bring new rows
    (flag 0 with id j inserts new_rows[j]); exact counts."""
    f = np.ascontiguousarray(flags, dtype=np.int32)
    i = np.ascontiguousarray(ids, dtype=np.int32)
    nr = np.ascontiguousarray(new_rows, dtype=np.float32)
    out = np.empty(int((f == 2).sum()) + 1, dtype=np.int32)
    nq = C.c_int(0)
    rc = lib().orc_update_run_rows(ds.ref, max_in_size, _iptr(f), _iptr(i), len(f), _fptr(nr), len(nr),
                                   C.c_float(r), _iptr(out), C.byref(nq))
    if rc != 0:
        raise RuntimeError(f"orc_update_run_rows failed: {rc}")
    return out[:nq.value]


def update_run(ds, p, max_in_size: int, flags, ids, r: float, exact: bool = False) -> np.ndarray:
    """Counts per query op; exact=True scans live rows instead of the
    reference's v1 tree search (which skips oversized last-level nodes)."""
    f = np.ascontiguousarray(flags, dtype=np.int32)
    i = np.ascontiguousarray(ids, dtype=np.int32)
    out = np.empty(int((f == 2).sum()) + 1, dtype=np.int32)
    nq = C.c_int(0)
    rc = lib().orc_update_run(ds.ref, C.byref(p), max_in_size, _iptr(f), _iptr(i), len(f),
                              C.c_float(r), 1 if exact else 0, _iptr(out), C.byref(nq))
    if rc != 0:
        raise RuntimeError(f"orc_update_run failed: {rc}")
    return out[:nq.value]
