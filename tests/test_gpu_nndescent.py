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


def _same_lists_up_to_ties(a_ids, a_d, a_cnt, b_ids, b_d, b_cnt, K, X):
    """Equal counts and bitwise-equal distances everywhere; ids equal except in
    runs of exactly equal distances, whose members may come in another order (the
    reference orders them by arrival in its sequential insertion, the device by
    id).  The run that a full list cuts at K may also keep another id of the same
    distance; its ids are checked to be at exactly that distance.  Returns the
    number of lists whose ids differ."""
    from oracle import ref
    assert np.array_equal(a_cnt, b_cnt)
    differ = 0
    for i in range(len(a_cnt)):
        c = int(a_cnt[i])
        da, db = a_d[i, :c].view(np.uint32), b_d[i, :c].view(np.uint32)
        assert np.array_equal(da, db), i
        if np.array_equal(a_ids[i, :c], b_ids[i, :c]):
            continue
        differ += 1
        s = 0
        while s < c:
            e = s + 1
            while e < c and da[e] == da[s]:
                e += 1
            if not np.array_equal(a_ids[i, s:e], b_ids[i, s:e]):
                assert e - s > 1, (i, s)  # a lone entry must match exactly
                if np.array_equal(np.sort(a_ids[i, s:e]), np.sort(b_ids[i, s:e])):
                    pass
                else:
                    assert e == c == K, (i, s)  # only the run cut at K may keep other ids
                    for j in range(s, e):
                        got = ref.l2(X[i], X[int(a_ids[i, j])])
                        assert np.float32(got).view(np.uint32) == da[j], (i, j)
            s = e
    return differ


@pytest.mark.skipif(not have_ref(), reason="reference library oracle/_ref not built")
def test_refine_matches_live_reference_d128(tmp_path):
    """Lists built by the reference's own parallel insertion (K > ef_construction,
    so lists start short), refined one iteration at a time on the device and by
    the one-thread restatement from the same state: equal up to the order of
    exactly equal distances.  (Each refineKNNG call starts with every entry new,
    hrnn.h:1742-1747, so one-iteration calls compare state for state.)"""
    from oracle import ref
    X = data.mixture(6000, 128, 24, 1.0, 5, 5)
    r = ref.RefIndex.create(128, 6000, 16, 60, 100, 80)
    r.add_points(X, threads=16)
    p = str(tmp_path / "pre.idx")
    r.save(p)
    Xs = idx.read_idx(p).vectors()
    ids, d, cnt = [np.ascontiguousarray(a).copy() for a in ref.RefIndex.load(p, 128).knng(80)]
    h = H.HRNN.load(p, 128)
    for _ in range(3):
        h.refineKNNG(1, 20)
        got = h.get_knng()
        flags = (np.arange(80)[None, :] < cnt[:, None]).astype(np.uint8)
        port.refine(Xs, ids, d, cnt, flags, 1, 20)
        _same_lists_up_to_ties(*got, ids, d, cnt, 80, Xs)
        ids, d, cnt = [np.ascontiguousarray(a).copy() for a in got]
    # recall against exact kNN (internal ids follow the parallel insertion order)
    Xd = Xs.astype(np.float64)
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


def test_refine_with_a_small_proposal_buffer_keeps_the_lists(monkeypatch):
    """A proposal buffer far smaller than one chunk's proposals: chunks overflow,
    are redone smaller (each retry at most a quarter of the one before) and the
    refinement ends with the lists of the unconstrained run, up to the order of
    exactly equal distances."""
    n, K = 20000, 60
    X = data.mixture(n, 128, 24, 1.0, 9, 9)
    h = H.HRNN(dim=128, max_elements=n, M=16, ef_construction=60, random_seed=100, K_knng=K)
    h.add_points(X)
    start = [np.ascontiguousarray(a).copy() for a in h.get_knng()]
    h.refineKNNG(2, 20)
    full = h.get_knng()
    h.set_knng(*start)
    monkeypatch.setenv("HRNN_REFINE_PCAP", "20000")
    h.refineKNNG(2, 20)
    small = h.get_knng()
    _same_lists_up_to_ties(*small, *full, K, X)
