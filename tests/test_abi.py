"""The C-ABI library: it loads, exports every declared symbol, parses the
reference file formats, and fails cleanly without a GPU (no compute here)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    syms = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gts_[a-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    lib = gts.lib_path()
    assert os.path.exists(lib), "libgts_b200.so is not built"
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = _declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    C.CDLL(lib)   # and it loads


def test_params_default_matches_reference():
    lib = gts._load_lib()
    p = gts.Params()
    lib.gts_params_default(C.byref(p))
    assert (p.tree_order, p.max_size, p.max_h, p.dis_code, p.infi_dis, p.max_in_size) == \
        (10, 20, 3, 100, 10000, 10)


def test_text_loaders_roundtrip(tmp_path):
    rows = G.gmm_rows(50, 7, 3, 0.5, 1)
    p = tmp_path / "d.txt"
    G.write_data_text(str(p), 2, rows=rows)
    d, n, m, r = gts.load(str(p))
    assert (d, n, m) == (7, 50, 2)
    np.testing.assert_allclose(r, rows, atol=1e-6)
    strs, lens = G.word_strings(30, 2)
    G.write_data_text(str(tmp_path / "s.txt"), 6, strs=strs, lens=lens)
    d, n, m, (s2, l2) = gts.load(str(tmp_path / "s.txt"))
    assert (n, m) == (30, 6)
    np.testing.assert_array_equal(l2, lens)
    np.testing.assert_array_equal(s2, strs)
    G.write_queries(str(tmp_path / "q.txt"), [3, 1, 4])
    assert gts.load_queries(str(tmp_path / "q.txt")).tolist() == [3, 1, 4]
    G.write_updates(str(tmp_path / "u.txt"), [0, 1, 2], [5, 6, 7])
    f, i = gts.load_updates(str(tmp_path / "u.txt"))
    assert f.tolist() == [0, 1, 2] and i.tolist() == [5, 6, 7]


def test_loader_errors(tmp_path):
    with pytest.raises(gts.GtsError) as e:
        gts.load(str(tmp_path / "missing.txt"))
    assert e.value.code == -4
    bad = tmp_path / "bad.txt"
    bad.write_text("3 2 2\n1 2 3\n4 5\n")
    with pytest.raises(gts.GtsError):
        gts.load(str(bad))
    long = tmp_path / "long.txt"
    long.write_text("1 1 6\n" + "a" * 200 + "\n")
    with pytest.raises(gts.GtsError):
        gts.load(str(long))


def test_reference_sample_parses():
    from tests.golden_io import sample_dir
    d = sample_dir()
    if d is None:
        pytest.skip("reference sample not present")
    dim, n, m, rows = gts.load(os.path.join(d, "sbw_example.txt"))
    assert (dim, n, m) == (300, 1000, 5)
    metric, rows2 = G.read_text_rows(os.path.join(d, "sbw_example.txt"))
    np.testing.assert_array_equal(rows, rows2)


def test_no_device_is_a_clean_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gts.GtsError) as e:
        gts.Index(np.zeros((10, 4), np.float32), 2)
    assert e.value.code == -2


def test_argument_checks_need_no_device():
    """Entry points reject bad arguments before touching a device."""
    lib = gts._load_lib()
    q = np.zeros(4, np.int32)
    out = np.zeros(4, np.int32)
    ip = q.ctypes.data_as(C.c_void_p)
    op = out.ctypes.data_as(C.c_void_p)
    # null handle, and a form the range entry point does not take
    assert lib.gts_range_form(None, ip, 4, C.c_float(1.0), 1, op) == -1
    assert lib.gts_range_form_device(None, ip, 4, C.c_float(1.0), 0, op, None) == -1
    assert lib.gts_plain_threads_set(None, 0, 256) == -1
    assert lib.gts_fast_config_set(None, 8, 0, 4, 16, 0) == -1
    msg = lib.gts_last_error()
    assert msg


def test_negative_scratch_budget_is_rejected_before_the_device():
    """gts_params.mem_budget_gb < 0 is an argument error (checked before any
    device work, so it fails the same way with or without a GPU)."""
    rows = G.gmm_rows(50, 4, 2, 0.5, 1)
    with pytest.raises(gts.GtsError) as e:
        gts.Index(rows, 2, mem_budget_gb=-1.0)
    assert e.value.code == -1 and "mem_budget_gb" in str(e.value)


def test_reference_compat_header_builds(tmp_path):
    """include/gts_ref_compat.h (the reference's entry points over this
    library) compiles as C++17 and links against libgts_b200 with the
    reference's call shapes (no GPU needed to build)."""
    src = tmp_path / "compat_main.cpp"
    src.write_text(r'''
#include "gts_ref/tree.cuh"
#include "gts_ref/file.cuh"
#include "gts_ref/search.cuh"
#include "gts_ref/update.cuh"
#include "gts_ref/search_v2.cuh"
#include "gts_ref/config.cuh"
int *data_info; short *data_d; char *data_s; int *size_s; int *qid_list; int qnum;
int *max_node_num; int *id_list; TN *node_list; int tree_h; int *empty_list;
int *qresult_count, *qresult_count_prefix, *result_id; float *result_dis;
int main(int argc, char **argv) {
    if (argc < 2) return 0;
    load(argv[1], data_info, data_d, data_s, size_s);
    loadQuery(argv[2], qid_list, qnum);
    indexConstru(data_d, data_s, size_s, data_info, id_list, node_list, max_node_num, tree_h, empty_list);
    searchIndexKnnV2(data_d, node_list, id_list, max_node_num, qid_list, qnum, 8, tree_h, data_info, empty_list, data_s, size_s);
    searchIndexRnnV2(data_d, node_list, id_list, max_node_num, qid_list, qnum, 1.f, tree_h, data_info, empty_list, data_s, size_s);
    float ts = 0; FILE *f = nullptr;
    searchIndexRnn(data_d, node_list, id_list, max_node_num, qid_list, qnum, 1.f, tree_h, data_info, empty_list,
                   qresult_count, qresult_count_prefix, result_id, result_dis, data_s, size_s, ts, f);
    searchIndexKnn(data_d, node_list, id_list, max_node_num, qid_list, qnum, 4, tree_h, data_info, empty_list,
                   result_id, result_dis, qresult_count, qresult_count_prefix, data_s, size_s, ts, f);
    loadUpdate(argv[3], update_list, update_num);
    float tu = 0; int cs = 0, cu = 0;
    updateIndexRnn(data_d, node_list, id_list, max_node_num, qid_list, 1, 1.f, tree_h, data_info, empty_list,
                   qresult_count, qresult_count_prefix, result_id, result_dis, data_s, size_s, f, ts, tu, cs, cu);
    saveK(argv[4], argv[5], result_id, result_dis, 4, qnum);
    return res[0] + (int)res_dis[0];
}
''')
    inc = os.path.join(ROOT, "include")
    libdir = os.path.dirname(gts.lib_path())
    cuda_inc = "/usr/local/cuda/include"
    cuda_lib = "/usr/local/cuda/lib64"
    if not os.path.isdir(cuda_inc):
        pytest.skip("CUDA headers not installed here")
    p = subprocess.run(["g++", "-std=c++17", "-I", inc, "-I", cuda_inc, str(src), "-o", str(tmp_path / "compat"),
                        "-L", libdir, "-lgts_b200", "-L", cuda_lib, "-lcudart"], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]
