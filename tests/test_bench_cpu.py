"""The bench's measurement helpers on the CPU: macro recall (queries with an empty
ground truth skipped, as utils.h:135-157 does) and the KNN-graph quality report."""
import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    argv, sys.argv = sys.argv, ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_macro_recall_skips_empty_ground_truth():
    b = _bench()
    gt = [np.array([1, 2, 3, 4], np.uint32), np.array([], np.uint32), np.array([7], np.uint32)]
    res = [np.array([1, 2], np.uint64), np.array([5], np.uint64), np.array([], np.uint64)]
    assert abs(b.macro_recall(gt, res) - (0.5 + 0.0) / 2) < 1e-12


def test_knng_quality_on_exact_and_damaged_lists():
    import torch
    b = _bench()
    rng = np.random.default_rng(3)
    X = rng.normal(size=(2000, 12)).astype(np.float32)
    K = 15
    D = ((X[:, None, :].astype(np.float64) - X[None]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    ids = np.argsort(D, 1)[:, :K].astype(np.uint32)
    d = np.take_along_axis(D, ids.astype(np.int64), 1).astype(np.float32)
    cnt = np.full(len(X), K, np.uint32)

    class Lists:
        def __init__(self, i, dd):
            self.i, self.dd = i, dd

        def get_knng(self):
            return self.i, self.dd, cnt

    q = b.knng_quality(torch, Lists(ids, d), X, K, torch.device("cpu"), sample=400)
    assert q["recall_at_K"] == 1.0 and q["dist_rel_err_max"] < 1e-6
    bad_i, bad_d = ids.copy(), d.copy()
    bad_i[:, -1] = (np.arange(len(X)) + 1000) % len(X)  # one wrong neighbour per list
    bad_d[:, -1] = D[np.arange(len(X)), bad_i[:, -1].astype(np.int64)].astype(np.float32)
    q2 = b.knng_quality(torch, Lists(bad_i, bad_d), X, K, torch.device("cpu"), sample=400)
    assert abs(q2["recall_at_K"] - (K - 1) / K) < 0.01


def test_workloads_are_well_formed():
    b = _bench()
    for name, W in b.WORKLOADS.items():
        assert W["n"] > 0 and W["d"] % 16 == 0 and W["K"] > 0 and W["k"] <= W["K"], name
        assert W["m_sweep"] == sorted(W["m_sweep"]), name
    assert "mixed-1M-d128-K500" in b.WORKLOADS


def test_ncu_traffic_is_tied_to_the_kernel_sources():
    """The captured DRAM bytes per unit scale with this launch's units, and are
    not reported once the kernel sources differ from the captured ones."""
    b = _bench()
    saved = dict(b.NCU_TRAFFIC)
    st = {"n_dist": 1_000_000, "n_posting": 3_000_000}
    try:
        b.NCU_TRAFFIC.clear()
        assert b.ncu_traffic("int8", "a", st)[0] is None
        b.NCU_TRAFFIC.update({"src_hash": b.search_src_hash(), "command": "c",
                              "per_unit": {("int8", "a"): 23.5, ("int8", "bc"): 25.0}})
        v, src = b.ncu_traffic("int8", "a", st)
        assert v == 23_500_000 and "c" in src and "beam distance" in src
        assert b.ncu_traffic("int8", "bc", st)[0] == 75_000_000
        assert b.ncu_traffic("fp32", "a", st)[0] is None
        b.NCU_TRAFFIC["src_hash"] = "0" * 16          # captured on other sources: not reported
        v, src = b.ncu_traffic("int8", "a", st)
        assert v is None and "predates" in src
    finally:
        b.NCU_TRAFFIC.clear()
        b.NCU_TRAFFIC.update(saved)
