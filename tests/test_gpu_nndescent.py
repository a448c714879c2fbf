"""GPU NNDescent (refineKNNG) against the reference run on one thread: the bulk
device iteration reproduces the single-thread reference's lists exactly."""
import numpy as np
import pytest

from conftest import have_ref
from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _same_lists(a_ids, a_d, a_cnt, b_ids, b_d, b_cnt):
    assert np.array_equal(a_cnt, b_cnt)
    for i in range(len(a_cnt)):
        c = int(a_cnt[i])
        assert np.array_equal(a_ids[i, :c], b_ids[i, :c]), i
        assert np.array_equal(a_d[i, :c].view(np.uint32), b_d[i, :c].view(np.uint32)), i


def test_refine_matches_single_thread_reference_golden(golden_idx, golden_refine):
    g = golden_refine
    h = H.HRNN.load(golden_idx, 32)
    h.set_knng(g["pre_ids"], g["pre_dists"], g["pre_cnt"])
    h.refineKNNG(int(g["iters"]), int(g["sample"]))
    ids, d, cnt = h.get_knng()
    _same_lists(ids, d, cnt, g["post_ids"], g["post_dists"], g["post_cnt"])


def test_refine_matches_oracle_nonfull_lists(golden_idx, golden_refine):
    """Lists shorter than K (the K > ef_construction case of the 1M build)."""
    g = golden_refine
    pre_cnt = np.minimum(g["pre_cnt"], 10).astype(np.uint32)
    h = H.HRNN.load(golden_idx, 32)
    h.set_knng(g["pre_ids"], g["pre_dists"], pre_cnt)
    h.refineKNNG(4, 9)
    ids, d, cnt = h.get_knng()
    oi, od, oc = g["pre_ids"].copy(), g["pre_dists"].copy(), pre_cnt.copy()
    flags = (np.arange(oi.shape[1])[None, :] < oc[:, None]).astype(np.uint8)
    port.refine(g["X"], oi, od, oc, flags, 4, 9)
    _same_lists(ids, d, cnt, oi, od, oc)


@pytest.mark.skipif(not have_ref(), reason="reference library oracle/_ref not built")
def test_refine_matches_live_reference_d128(tmp_path):
    from oracle import ref
    X = data.mixture(6000, 128, 24, 1.0, 5, 5)
    r = ref.RefIndex.create(128, 6000, 16, 60, 100, 80)   # K > ef_construction: lists start short
    r.add_points(X, threads=16)
    p = str(tmp_path / "pre.idx")
    r.save(p)
    r.refine(3, 20, threads=1)
    exp = r.knng(80)
    h = H.HRNN.load(p, 128)
    h.refineKNNG(3, 20)
    got = h.get_knng()
    _same_lists(*got, *exp)
    # recall against exact kNN (internal ids follow the parallel insertion order)
    Xd = idx.read_idx(p).vectors().astype(np.float64)
    nx = (Xd * Xd).sum(1)
    D = nx[:500, None] - 2 * Xd[:500] @ Xd.T + nx[None, :]
    D[np.arange(500), np.arange(500)] = np.inf
    exact = np.argsort(D, axis=1)[:, :80]
    rec = np.mean([len(np.intersect1d(exact[i], got[0][i, :got[2][i]])) / 80 for i in range(500)])
    assert rec > 0.9


@pytest.mark.parametrize("K", [30, 7])
def test_refine_odd_list_widths_match_oracle(golden_refine, tmp_path, K):
    """K_knng values whose per-warp merge buffer is not a multiple of 8 bytes
    before rounding (K * 18 % 8 != 0)."""
    g = golden_refine
    X = g["X"]
    n = X.shape[0]
    w = min(K, g["pre_ids"].shape[1])
    ids = np.zeros((n, K), np.uint32)
    d = np.zeros((n, K), np.float32)
    ids[:, :w] = g["pre_ids"][:, :w]
    d[:, :w] = g["pre_dists"][:, :w]
    cnt = np.minimum(g["pre_cnt"], w).astype(np.uint32)
    p = str(tmp_path / f"k{K}.idx")
    idx.write_idx(p, X, ids, d, cnt, M=8)
    h = H.HRNN.load(p, X.shape[1])
    h.refineKNNG(3, 10)
    got = h.get_knng()
    oi, od, oc = ids.copy(), d.copy(), cnt.copy()
    flags = (np.arange(K)[None, :] < oc[:, None]).astype(np.uint8)
    port.refine(X, oi, od, oc, flags, 3, 10)
    _same_lists(*got, oi, od, oc)
