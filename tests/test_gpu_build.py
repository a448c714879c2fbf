"""GPU index construction (batched HNSW insertion + KNN seed, NNDescent, CSR) and
the reference reading the result: the .idx written after a GPU build is a valid
reference index, and the reference's own searchRknn on it returns the GPU's
answers."""
import numpy as np
import pytest

from conftest import have_ref
from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def built(tmp_path_factory):
    X = data.mixture(20000, 128, 32, 1.0, 21, 21)
    Q = data.mixture(300, 128, 32, 1.0, 21, 22)
    h = H.HRNN(128, 20000, 16, 100, 100, 64)
    h.add_points(X)
    seed = h.get_knng()
    h.refineKNNG(4, 20)
    h.buildRKNNG()
    p = str(tmp_path_factory.mktemp("b") / "gpu.idx")
    h.saveIndex(p)
    return X, Q, h, p, seed


def test_graph_invariants(built):
    X, Q, h, p, seed = built
    f = idx.read_idx(p)
    assert f.n == 20000 and f.knng_built and f.rknng_built
    adj = f.adj0()
    cnt = adj[:, 0] & 0xFFFF
    assert cnt.max() <= 32 and cnt.min() >= 1
    for i in range(0, 20000, 97):
        nb = adj[i, 1:1 + cnt[i]]
        assert i not in nb and len(set(nb.tolist())) == len(nb) and nb.max() < 20000
    lv = f.levels()
    assert lv[f.enterpoint] == f.maxlevel == lv.max()
    # KNN seed: ascending exact distances, no self, no duplicates
    ids, d, c = seed
    rows = np.arange(1, 20000, 211)   # element 0 is inserted first, with no seed (hrnn.h:1505-1509)
    for i in rows:
        k = int(c[i])
        assert 0 < k <= 64 and i not in ids[i, :k] and len(set(ids[i, :k].tolist())) == k
        assert np.all(np.diff(d[i, :k]) >= 0)
        exact = port.l2_batch(np.repeat(f.vectors()[i:i + 1], k, 0), f.vectors()[ids[i, :k]])
        assert np.array_equal(exact.view(np.uint32), d[i, :k].view(np.uint32))


def test_knn_graph_recall(built):
    X, Q, h, p, _ = built
    ids, d, c = h.get_knng()
    Xd = X.astype(np.float64)
    nx = (Xd * Xd).sum(1)
    rows = np.arange(0, 20000, 40)
    D = nx[rows, None] - 2 * Xd[rows] @ Xd.T + nx[None, :]
    D[np.arange(len(rows)), rows] = np.inf
    exact = np.argsort(D, axis=1)[:, :64]
    rec = np.mean([len(np.intersect1d(exact[j], ids[r, :c[r]])) / 64 for j, r in enumerate(rows)])
    assert rec > 0.97, rec


def test_rknn_recall_against_fp64_gt(built):
    X, Q, h, p, _ = built
    kth = data.kth_nn_fp64(X, 10)
    gt = data.rknn_gt_fp64(X, Q, kth)
    res = h.search_rknn_batch(Q, 10, 64, 100, threshold=1.0, k=10)
    assert data.macro_recall(gt, res) > 0.95


def test_search_on_gpu_index_matches_oracle(built):
    X, Q, h, p, _ = built
    O = port.OracleIndex(idx.read_idx(p))
    for m, kp, ef in ((3, 64, 50), (10, 32, 100)):
        a = h.search_rknn_batch(Q, m, kp, ef, k=10)
        b = O.search_batch(Q, m, kp, ef, k=10)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.skipif(not have_ref(), reason="reference library oracle/_ref not built")
def test_reference_reads_gpu_index(built):
    from oracle import ref
    X, Q, h, p, _ = built
    r = ref.RefIndex.load(p, 128)
    assert r.count() == 20000
    a = r.search_batch(Q, 10, 64, 100, k=10)
    b = h.search_rknn_batch(Q, 10, 64, 100, k=10)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_large_answer_sets_match_oracle(built):
    """k = K_knng and many proxies: answer sets of hundreds to thousands of points
    (exercises the overflow path of the shared-memory phase B/C kernel)."""
    X, Q, h, p, _ = built
    O = port.OracleIndex(idx.read_idx(p))
    for m, kp, k, th in ((50, 64, 64, 1.0), (40, 64, 64, 2.0), (30, 16, 40, 1.0)):
        a = h.search_rknn_batch(Q[:60], m, kp, 100, threshold=th, k=k)
        b = O.search_batch(Q[:60], m, kp, 100, threshold=th, k=k)
        assert all(np.array_equal(x, y) for x, y in zip(a, b)), (m, kp, k, th)
    assert max(len(x) for x in a) > 100


@pytest.mark.parametrize("prec", [H.PREC_BF16, H.PREC_INT8])
def test_mixed_precision_decisions_and_recall(built, prec):
    """BF16 (or INT8) beam + BF16-screened verification: every returned point
    passes the exact FP32 test (or the FP64 test inside the tie band), and recall
    stays at the plain form's level."""
    X, Q, h, p, _ = built
    f = idx.read_idx(p)
    V = f.vectors()
    ids, d, cnt = f.knng()
    lab2id = {int(l): i for i, l in enumerate(f.labels())}
    kth = data.kth_nn_fp64(X, 10)
    gt = data.rknn_gt_fp64(X, Q, kth)
    plain = h.search_rknn_batch(Q, 10, 64, 100, k=10)
    try:
        h.set_precision(prec)
        mixed = h.search_rknn_batch(Q, 10, 64, 100, k=10)
        st = h.last_search_stats()
    finally:
        h.set_precision(H.PREC_FP32_EXACT)
    assert st["n_lowp_decided"] > 0.9 * (st["n_lowp_decided"] + st["n_fp32_decided"])
    bad = 0
    for qi, res in enumerate(mixed):
        for lab in res:
            i = lab2id[int(lab)]
            d32 = port.l2(Q[qi], V[i])
            kd = d[i, 9] if cnt[i] > 9 else np.float32(np.finfo(np.float32).max)
            bad += not (d32 <= kd)
    assert bad <= st["n_fp64_flipped"]
    assert data.macro_recall(gt, mixed) >= data.macro_recall(gt, plain) - 0.01
