"""The C++ drivers end to end on a small mixture: the float64 ground-truth tool,
hrnn_build, hrnn_search (its recall equals the Python API's on the same index,
one query per call or all at once) and hrnn_dynamic_test."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from oracle import data, idx

import hrnn_b200 as H
from hrnn_b200 import groundtruth as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "hrnn_b200", "drivers", "bin")


def run(name, *args):
    r = subprocess.run([os.path.join(BIN, name), *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def recalls(out):
    return [float(x) for x in re.findall(r"Macro Recall = ([0-9.]+)", out)]


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("drv")
    X = data.mixture(3000, 32, 10, 1.0, 41, 41)
    Q = data.mixture(120, 32, 10, 1.0, 41, 42)
    base, query, gt = str(d / "base.fbin"), str(d / "query.fbin"), str(d / "gt.bin")
    G.write_fbin(base, X)
    G.write_fbin(query, Q)
    r = subprocess.run([sys.executable, "-m", "hrnn_b200.groundtruth", "--base", base, "--query", query, "--k", "10",
                        "--output", gt], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return X, Q, base, query, gt, str(d / "index.idx")


def test_build_then_search(files):
    X, Q, base, query, gt, index = files
    run("hrnn_build", "--base", base, "--index_path", index, "--M", 8, "--ef_construction", 64, "--K_knng", 40,
        "--nn_iters", 2, "--nn_sample", 12)
    f = idx.read_idx(index)
    assert f.n == 3000 and f.knng_built and f.rknng_built
    out = run("hrnn_search", "--index_path", index, "--query", query, "--gt", gt, "--k", 10, "--K_prime", 40,
              "--m", "3,8", "--ef_search", 60)
    r_all = recalls(out)
    out1 = run("hrnn_search", "--index_path", index, "--query", query, "--gt", gt, "--k", 10, "--K_prime", 40,
               "--m", "3,8", "--ef_search", 60, "--batch", 1)
    assert recalls(out1) == r_all
    # the Python API on the same file and ground truth
    h = H.HRNN.load(index, 32)
    g = G.read_rknn_gt(gt)
    exp = []
    for m in (3, 8):
        res = h.search_rknn_batch(Q, m, 40, 60, threshold=1.0, k=10)
        rs = [len(np.intersect1d(ids, r)) / len(ids) for (ids, _), r in zip(g, res) if len(ids)]
        exp.append(float(np.mean(rs)))
    assert all(abs(a - b) <= 1e-6 for a, b in zip(r_all, exp)), (r_all, exp)
    assert r_all[1] > 0.8
    outb = run("hrnn_search", "--index_path", index, "--query", query, "--gt", gt, "--k", 10, "--K_prime", 40,
               "--m", 8, "--ef_search", 60, "--precision", "bf16")
    assert abs(recalls(outb)[0] - r_all[1]) < 0.02


def test_dynamic_driver(files):
    X, Q, base, query, gt, _ = files
    out = run("hrnn_dynamic_test", "--base", base, "--query", query, "--gt", gt, "--M", 8, "--ef_construction", 64,
              "--K_knng", 40, "--nn_iters", 2, "--nn_sample", 12, "--m", 8, "--ef_search", 60, "--m_update", 4)
    assert "Index size after maintenance: 3000" in out
    r = recalls(out)
    assert r and r[-1] > 0.7, out[-1500:]
