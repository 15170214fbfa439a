"""The drop-in command line: same argument order and result-file layout as
the reference's bin/GTS (src/main.cu:43-180), values from the library."""
import os
import subprocess

import numpy as np
import pytest

import gts_b200 as gts
from gts_b200 import datagen as G
from tests import golden_io as GI

pytestmark = pytest.mark.gpu
CLI = os.path.join(os.path.dirname(gts.lib_path()), "gts")


def _run(args):
    p = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    return p.stdout


def test_cli_knn_range_update(tmp_path):
    rows = G.gmm_rows(3000, 16, 8, 0.3, 31)
    qids = G.query_ids(3000, 77, 32)
    data = tmp_path / "d.txt"
    G.write_data_text(str(data), 2, rows=rows)
    G.write_queries(str(tmp_path / "q.txt"), qids)
    _, _, _, parsed = gts.load(str(data))
    with gts.Index(parsed, 2, max_h=4) as idx:
        want_k = idx.knn(qids, 6)
        want_r = idx.range(qids, 1.5)
    out = tmp_path / "k.txt"
    _run([data, tmp_path / "q.txt", 0, 6, out, "--max-h", 4, "--ids", tmp_path / "kk"])
    head, vals, tail = GI.parse_result_file(str(out))
    assert head == "Knn search num: 6"
    assert vals == [f"{v:f}" for v in want_k]
    assert tail[0].startswith("Time of index construction: ") and tail[1].startswith("Search time: ")
    ids = np.loadtxt(tmp_path / "kk.ids", dtype=np.int64, ndmin=2)
    assert ids.shape == (77, 6) and (ids[:, 0] == qids).all()
    out = tmp_path / "r.txt"
    _run([data, tmp_path / "q.txt", 1, 1.5, out, "--max-h", 4, "--form", "fast"])
    head, vals, _ = GI.parse_result_file(str(out))
    assert head == "Range search radius: 1.500000"
    assert vals == [str(v) for v in want_r]
    flags, uids = G.update_stream(3000, 120, 33)
    G.write_updates(str(tmp_path / "u.txt"), flags, uids)
    out = tmp_path / "u_out.txt"
    _run([data, tmp_path / "u.txt", 2, 1.5, out, "--max-h", 4])
    head, vals, tail = GI.parse_result_file(str(out))
    assert head == "Range search radius (check for updates): 1.500000"
    assert len(vals) == int((flags == 2).sum())
    assert tail[2].startswith("Search time in update : ")


def test_cli_on_reference_sample(tmp_path):
    d = GI.sample_dir()
    if d is None or not os.path.exists(os.path.join(GI.GOLDEN, "sample_knn_k8.txt")):
        pytest.skip("reference sample data or its golden results not present")
    runs = [("0", "8", "sample_knn_k8.txt", "sbw_example_qid.txt"),
            ("1", "30", "sample_range_r30.txt", "sbw_example_qid.txt"),
            ("2", "59", "sample_update_r59.txt", "sbw_example_u.txt")]
    for op, par, gold, qf in runs:
        out = tmp_path / gold
        _run([os.path.join(d, "sbw_example.txt"), os.path.join(d, qf), op, par, out])
        got = open(out).read().split("\n")[:3]
        want = open(os.path.join(GI.GOLDEN, gold)).read().split("\n")[:3]
        assert got == want, gold


def test_reference_main_over_the_compat_headers(tmp_path):
    """The reference's own src/main.cu, unmodified, compiled against
    include/gts_ref (its entry points over this library; built by
    `make -C oracle ref` where the checkout is) gives the reference's result
    files on the reference's sample: kNN, range and the update stream."""
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "GTS_compat")
    d = GI.sample_dir()
    if d is None or not os.path.exists(exe):
        pytest.skip("the reference's sample or its main.cu build over the compat headers is not present")
    runs = [("0", "8", "sample_knn_k8.txt", "sbw_example_qid.txt"),
            ("0", "20", "sample_knn_k20.txt", "sbw_example_qid.txt"),
            ("1", "30", "sample_range_r30.txt", "sbw_example_qid.txt"),
            ("2", "59", "sample_update_r59.txt", "sbw_example_u.txt")]
    for op, par, gold, qf in runs:
        out = tmp_path / gold
        p = subprocess.run([exe, os.path.join(d, "sbw_example.txt"), os.path.join(d, qf), op, par, str(out)],
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        got = open(out).read().split("\n")
        want = open(os.path.join(GI.GOLDEN, gold)).read().split("\n")
        assert got[:3] == want[:3], gold
        # the timing lines of main.cu's layout follow
        assert got[3].startswith("Time of index construction: "), gold
