"""gts_knn_device_noalloc through the C ABI: the same answers as
gts_knn_device's GTS_FORM_FAST (bit-identical, the tolerance of every kNN
parity test here), on two calls in a row, plus its size limit."""
import ctypes as C

import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

pytestmark = pytest.mark.gpu

MAX_QUERIES = 512


def _knn(lib, fn, h, q, k, torch, form=None):
    dq = torch.from_numpy(q).cuda()
    kth = torch.full((len(q),), -1.0, dtype=torch.float32, device="cuda")
    ids = torch.full((len(q) * k,), -7, dtype=torch.int32, device="cuda")
    dis = torch.full((len(q) * k,), -1.0, dtype=torch.float32, device="cuda")
    args = [h, C.c_void_p(dq.data_ptr()), len(q), k]
    if form is not None:
        args.append(form)
    args += [C.c_void_p(kth.data_ptr()), C.c_void_p(ids.data_ptr()), C.c_void_p(dis.data_ptr()),
             C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    rc = fn(*args)
    assert rc == 0, lib.gts_last_error().decode()
    torch.cuda.synchronize()
    return kth.cpu().numpy(), ids.cpu().numpy().reshape(len(q), k), dis.cpu().numpy().reshape(len(q), k)


def test_noalloc_matches_fast_form_twice():
    torch = pytest.importorskip("torch")
    lib = gts._load_lib()
    rows = G.gmm_rows(20000, 128, 32, 0.2, seed=31)
    calls = [(G.query_ids(20000, 500, seed=32), 8), (G.query_ids(20000, MAX_QUERIES, seed=33), 33)]
    with gts.Index(rows, 2, max_h=5) as idx:
        h = idx._h
        want = [_knn(lib, lib.gts_knn_device, h, q, k, torch, form=gts.FORM_FAST) for q, k in calls]
        for (q, k), w in zip(calls, want):
            got = _knn(lib, lib.gts_knn_device_noalloc, h, q, k, torch)
            for x, y in zip(got, w):
                np.testing.assert_array_equal(x, y, err_msg=f"k={k}")


def test_noalloc_rejects_oversize_batch():
    torch = pytest.importorskip("torch")
    lib = gts._load_lib()
    rows = G.gmm_rows(3000, 32, 4, 0.5, seed=34)
    with gts.Index(rows, 2, max_h=4) as idx:
        h = idx._h
        q = G.query_ids(3000, 8, seed=35)
        _knn(lib, lib.gts_knn_device, h, q, 4, torch, form=gts.FORM_FAST)
        dq = torch.zeros(MAX_QUERIES + 1, dtype=torch.int32, device="cuda")
        out = torch.zeros(MAX_QUERIES + 1, dtype=torch.float32, device="cuda")
        rc = lib.gts_knn_device_noalloc(h, C.c_void_p(dq.data_ptr()), MAX_QUERIES + 1, 4,
                                        C.c_void_p(out.data_ptr()), None, None, None)
        assert rc == -1  # GTS_ERR_INVALID
        assert b"exceed the maximum of 512" in lib.gts_last_error()


def test_noalloc_equals_the_oracle_and_answers_overflowed_lists(oracle):
    """Against exact brute force directly: 1,500 copies of one row make the
    candidate list of every query among them overflow (every copy is at
    distance 0), so the entry point's plain-traversal fallback answers
    those; the other queries come from the filter.  Two calls in a row."""
    torch = pytest.importorskip("torch")
    lib = gts._load_lib()
    base = G.gmm_rows(6000, 64, 8, 0.3, seed=36)
    rows = np.concatenate([base, np.repeat(base[7:8], 1500, axis=0)])
    ds = oracle.Dataset(2, rows)
    q = np.concatenate([np.array([7, 6000, 6500, 7499], np.int32), G.query_ids(6000, 200, seed=37)])
    with gts.Index(rows, 2, max_h=4) as idx:
        idx.prepare(gts.FORM_FAST)
        for k in (8, 20):
            kth, ids, dis = _knn(lib, lib.gts_knn_device_noalloc, idx._h, q, k, torch)
            assert idx.search_stats()["fallback"] >= 4     # the copies' lists overflowed
            bk, bi, bd = oracle.knn_brute(ds, q, k)
            np.testing.assert_array_equal(ids, bi, err_msg=f"k={k}")
            np.testing.assert_array_equal(kth, bk, err_msg=f"k={k}")
            np.testing.assert_array_equal(dis, bd, err_msg=f"k={k}")
