"""Loading of the golden fixtures produced by tests/golden/make_fixtures.py."""
import glob
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_case(name):
    """-> (case dict, data, qids, radii, fixture)  with data regenerated from seeds."""
    from tests.golden.make_fixtures import make_case_data
    fx = dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    c = json.loads(str(fx["case"]))
    data, digest, qids, radii, upd = make_case_data(c)
    assert digest == str(fx["digest"]), f"{name}: regenerated data differs from the fixture"
    assert np.array_equal(qids, fx["qids"])
    return c, data, qids, radii, fx


def sample_dir():
    """Directory holding the reference's sample data set, if present here:
    the copy the oracle's reference build stages (oracle/_ref/sample, made by
    `make -C oracle ref`), or the checkout named by $GTS_REF_DIR."""
    ref = os.environ.get("GTS_REF_DIR", "")
    for d in (os.environ.get("GTS_SAMPLE_DIR", ""), os.path.join(GOLDEN, "..", "..", "oracle", "_ref", "sample"),
              os.path.join(ref, "Datasets Sample") if ref else ""):
        if d and os.path.exists(os.path.join(d, "sbw_example.txt")):
            return d
    return None


def parse_result_file(path):
    """main.cu result layout -> (header line, values list, trailer lines)."""
    with open(path) as f:
        lines = f.read().split("\n")
    return lines[0], lines[2].split(), lines[3:]
