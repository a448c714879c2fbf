"""Batched insertPointDynamic on the GPU (hrnn.h:2360-2534): list invariants with
exact FP32 distances, KNN-graph recall against brute force next to the
reference's own insertPointDynamic on the same points, and searches on the
maintained index that match the oracle bit for bit."""
import numpy as np
import pytest

from conftest import have_ref
from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu

N0, N1, D, K = 4000, 2000, 64, 40


def _data():
    X = data.mixture(N0 + N1, D, 24, 1.0, 31, 31)
    Q = data.mixture(200, D, 24, 1.0, 31, 32)
    return X, Q


def _knn_recall(ids, cnt, X, rows, k):
    Xd = X.astype(np.float64)
    nx = (Xd * Xd).sum(1)
    Dm = nx[rows, None] - 2 * Xd[rows] @ Xd.T + nx[None, :]
    Dm[np.arange(len(rows)), rows] = np.inf
    exact = np.argsort(Dm, 1)[:, :k]
    hit = [len(set(exact[r].tolist()) & set(ids[i, :min(k, int(cnt[i]))].tolist())) / k for r, i in enumerate(rows)]
    return float(np.mean(hit))


def _build(X):
    h = H.HRNN(D, N0 + N1, 8, 64, 100, K)
    h.add_points(X[:N0], np.arange(N0, dtype=np.uint64))
    h.refineKNNG(3, 16)
    h.buildRKNNG_mutable()
    return h


@pytest.mark.parametrize("m_update,bidir", [(0, False), (6, True)])
def test_dynamic_insert_lists_and_recall(tmp_path, m_update, bidir):
    X, Q = _data()
    h = _build(X)
    h.insertPointDynamic(X[N0:], np.arange(N0, N0 + N1, dtype=np.uint64), m_update, bidir)
    st = h.last_dynamic_stats()
    assert st["n_inserted"] == N1 and st["n_batches"] >= 1 and st["n_dist"] > 0 and st["n_updates"] > 0
    assert h.getCurrentElementCount() == N0 + N1 and h.rknng_built_
    ids, dist, cnt = h.get_knng()
    p = str(tmp_path / "dyn.idx")
    h.saveIndex(p)
    f = idx.read_idx(p)
    V = f.vectors()
    for i in range(0, N0 + N1, 53):
        c = int(cnt[i])
        assert 0 < c <= K and i not in ids[i, :c] and len(set(ids[i, :c].tolist())) == c
        assert np.all(np.diff(dist[i, :c]) >= 0)
        exact = port.l2_batch(np.repeat(V[i:i + 1], c, 0), V[ids[i, :c]])
        assert np.array_equal(exact.view(np.uint32), dist[i, :c].view(np.uint32)), i
    rows = np.arange(0, N0 + N1, 7)
    rec = _knn_recall(ids, cnt, X, rows, 10)
    # the new points' lists are HNSW seeds (ef_construction = 64), refined only
    # with `bidirectional`: the bar is the reference's own result below
    assert rec > 0.6, rec
    if have_ref():
        from oracle import ref
        r = ref.RefIndex.create(D, N0 + N1, 8, 64, 100, K)
        r.add_points(X[:N0], np.arange(N0, dtype=np.uint64))
        r.refine(3, 16)
        r.build_mutable()
        r.insert_dynamic(X[N0:], np.arange(N0, N0 + N1, dtype=np.uint64), m_update, bidir)
        rids, _, rcnt = r.knng(K)
        rrec = _knn_recall(rids, rcnt, X, rows, 10)
        print(f"KNN recall@10 after inserts: GPU {rec:.4f}, reference {rrec:.4f}")
        assert rec >= rrec - 0.02, (rec, rrec)
    # search on the maintained index: bit-identical to the oracle on the same file
    O = port.OracleIndex(f)
    got = h.search_rknn_batch(Q, 8, K, 60, threshold=1.0, k=10)
    exp = O.search_batch(Q, 8, K, 60, threshold=1.0, k=10)
    assert all(np.array_equal(a, b) for a, b in zip(got, exp))


def test_dynamic_insert_reverse_lists_exact():
    """After the inserts the reverse lists are exactly the transpose of the lists."""
    X, _ = _data()
    h = _build(X)
    h.insertPointDynamic(X[N0:N0 + 500], np.arange(N0, N0 + 500, dtype=np.uint64), 4, False)
    ids, _, cnt = h.get_knng()
    off, ent, rb, wide = h.get_rknng()
    n = N0 + 500
    owners = (ent >> np.uint64(rb)) if wide else (ent >> np.uint32(rb))
    for y in range(0, n, 37):
        got = sorted(int(o) for o in owners[off[y]:off[y + 1]])
        exp = sorted(i for i in range(n) if y in ids[i, :cnt[i]])
        assert got == exp, y


def test_dynamic_insert_errors():
    X, _ = _data()
    h = H.HRNN(D, N0 + 10, 8, 64, 100, K)
    h.add_points(X[:N0])
    h.refineKNNG(1, 8)
    with pytest.raises(H.HrnnError):  # buildRKNNG_mutable not called
        h.insertPointDynamic(X[N0:N0 + 5], np.arange(N0, N0 + 5, dtype=np.uint64))
    h.buildRKNNG_mutable()
    with pytest.raises(H.HrnnError):  # beyond max_elements
        h.insertPointDynamic(X[N0:N0 + 20], np.arange(N0, N0 + 20, dtype=np.uint64))
    h.insertPointDynamic(X[N0:N0 + 10], np.arange(N0, N0 + 10, dtype=np.uint64))
    assert h.getCurrentElementCount() == N0 + 10


@pytest.mark.parametrize("m_update,bidir", [(4, False), (0, True)])
def test_mutable_reverse_lists_follow_the_graph(m_update, bidir):
    """The device's mutable reverse lists (buildRKNNG_mutable, edited in place by
    every insert batch: the new points join their neighbours' lists, accepted and
    pushed-out entries move) equal the transpose of the KNN graph after each call,
    as sets, for every element."""
    X, _ = _data()
    h = _build(X)

    def check():
        ids, _, cnt = h.get_knng()
        lists = h.get_rknng_mutable()
        n = h.getCurrentElementCount()
        exp = [[] for _ in range(n)]
        for i in range(n):
            for y in ids[i, :cnt[i]]:
                exp[int(y)].append(i)
        bad = [y for y in range(n) if sorted(lists[y].tolist()) != sorted(exp[y])]
        assert not bad, bad[:5]

    check()
    for a, b in ((N0, N0 + 700), (N0 + 700, N0 + N1)):
        h.insertPointDynamic(X[a:b], np.arange(a, b, dtype=np.uint64), m_update, bidir)
        check()
